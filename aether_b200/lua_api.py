"""Scripting front end with the reference's Lua method names.

The reference drives this path from Lua scripts: ``MODE("fdtd_normal")``,
``Structure(...)``, ``Material()``, ``create_sensor(...)``,
``create_source(...)`` and their methods (src/finite_differences/FDTD/modes/
lua_fdtd.cpp:363-411, src/finite_differences/core/lua_fd.cpp, src/structure/
lua_structure.cpp:292-548, src/finite_differences/FDTD/sensors/
lua_sensors.cpp:26-147, src/finite_differences/FDTD/sources/lua_sources.cpp,
src/materials/lua_material.cpp:380-412). This module offers the same objects
and method names in Python, so a script ports line by line:

    mat = Material(); mat.refractive_index(1.5)
    s = Structure(lambda st: (st.size(300e-9, 300e-9, 150e-9),
                              st.default_material(0),
                              st.add_layer("Z", 0, 50e-9, 1)))
    f = MODE("fdtd_normal"); f.structure(s); f.Dxyz(5e-9); f.N_tsteps(20000)
    f.spectrum(1000e-9, 2000e-9, 2001); f.pml_zp(25, 25, 1, 0.2)
    f.material(0, Material()); f.material(1, mat)
    out = f.compute()

Structure scripts (Lua files in the reference) become Python callables that
receive the Structure: they set its lx, ly, lz (the Lua globals of the same
names) and call its add_* methods; declare_parameter returns the parameter's
current value (the reference sets a Lua global). As in the reference,
Structure.parameter(name, value) only records the value, and the script is
evaluated again by Structure.finalize(), which Mode.structure() calls
(FD_Mode::set_structure, lua_fd.cpp:465-469).

compute() runs the mode's driver on the GPU through the C ABI and returns the
driver's results instead of writing its files: normal incidence the
spectdata_norm / spectdata_norm2 columns, oblique incidence the obl_ rows per
wavevector, and every registered sensor's flux, DFT or map in registration
order.

Not available: Lua material files (Material.load_script, material(i, "file");
describe the model with the add_* terms) and add_lua_def (a Lua function per
point)."""
from __future__ import annotations

import ctypes as C
import math
import time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import _abi as A
from . import fdtd
from . import oblique as OBL
from ._lib import check, load
from .scene import Scene


def nearest_integer(x: float) -> int:
    """mathUT.cpp:1169-1173."""
    return int(x + 0.5) if x >= 0 else int(x - 0.5)


# ---- materials --------------------------------------------------------------

class Material:
    """Material() with the FDTD-compatible models (material.h:33-93)."""

    def __init__(self):
        self.eps_inf = 1.0
        self.terms = {"debye": [], "drude": [], "lorentz": [], "critpoint": []}
        self._name = ""

    def refractive_index(self, n: float):
        self.eps_inf = float(n) * float(n)

    def epsilon_infinity(self, eps: float):
        self.eps_inf = float(eps)

    epsilon_infty = epsilon_infinity

    def add_debye(self, ds, t0):
        self.terms["debye"].append((ds, t0))

    def add_drude(self, wd, g):
        self.terms["drude"].append((wd, g))

    def add_lorentz(self, a, o, g):
        self.terms["lorentz"].append((a, o, g))

    def add_crit_point(self, a, o, p, g):
        self.terms["critpoint"].append((a, o, p, g))

    def name(self, s: str):
        self._name = s

    description = name

    def load_script(self, path: str, search=()):
        """Material:load_script (lua_material.cpp:365-373, Loader::load
        :466-497): resets the material and runs a material file of the
        reference's library format (mat_lib/*.lua) with aether_b200.matlib's
        reader. `path` is found as written, else in each directory of
        `search` (PathManager::locate_file's order, filehdl.cpp:292-340:
        working directory, then the calling script's directory, ...)."""
        from . import matlib
        m = matlib.load_file(locate_file(path, search))
        self.eps_inf = m.eps_inf
        self.terms = {k: list(v) for k, v in m.terms.items()}
        self._name = m.name
        self._refusal = m.refusal()

    def desc(self) -> A.MaterialDesc:
        why = getattr(self, "_refusal", None)
        if why:
            raise ValueError(f"material {self._name!r} cannot be used by the FDTD: {why}")
        t = self.terms
        return A.material_desc(self.eps_inf, debye=t["debye"], drude=t["drude"], lorentz=t["lorentz"],
                               critpoint=t["critpoint"])


def locate_file(path: str, search=()) -> str:
    """PathManager::locate_file (filehdl.cpp:292-340) over the given
    directories: an absolute path must exist; a relative one is tried from
    the working directory, then from each directory of `search`."""
    import os
    if os.path.isabs(path):
        if not os.path.exists(path):
            raise FileNotFoundError(f"couldn't locate absolute path {path!r}")
        return path
    for d in (os.getcwd(),) + tuple(search):
        cand = os.path.normpath(os.path.join(d, path))
        if os.path.exists(cand):
            return cand
    raise FileNotFoundError(f"couldn't locate {path!r}")


def const_material(n: float) -> Material:
    m = Material()
    m.refractive_index(n)
    return m


# ---- structures -------------------------------------------------------------

class _MT19937:
    """The 32-bit Mersenne Twister (Matsumoto and Nishimura, 1998) with the
    standard integer seeding, i.e. std::mt19937(seed)."""

    def __init__(self, seed):
        self.mt = [0] * 624
        self.mt[0] = seed & 0xFFFFFFFF
        for i in range(1, 624):
            self.mt[i] = (1812433253 * (self.mt[i - 1] ^ (self.mt[i - 1] >> 30)) + i) & 0xFFFFFFFF
        self.i = 624

    def __call__(self):
        if self.i >= 624:
            mt = self.mt
            for k in range(624):
                y = (mt[k] & 0x80000000) | (mt[(k + 1) % 624] & 0x7FFFFFFF)
                mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
            self.i = 0
        y = self.mt[self.i]
        self.i += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        return y ^ (y >> 18)


def random_packing(x_max, y_max, r, n_part, seed=None, max_iterations=1000000):
    """random_packing(x_max, y_max, r, N[, seed]) of the structure scripts
    (lua_structure.cpp, random_packing; phys_tools.cpp:244-426): N discs of
    radius r in a periodic x_max x y_max cell, particle 0 fixed at the origin,
    the others drawn from std::mt19937(seed) and pushed apart by soft
    repulsion until no particle moves (the reference's loop has no bound; here
    it stops with an error after max_iterations). Returns the x and y lists."""
    import time as _time
    gen = _MT19937(int(_time.time()) if seed is None or seed < 0 else int(seed))
    span = 4294967295.0   # gen.max() - gen.min()
    px, py = [0.0] * n_part, [0.0] * n_part
    for i in range(1, n_part):
        # set(randp(x_max, gen), randp(y_max, gen), r): the reference's x86-64
        # GCC build evaluates these arguments right to left, so y is drawn first
        py[i] = y_max * gen() / span
        px[i] = x_max * gen() / span
    stable = [False] * n_part
    fx, fy = [0.0] * n_part, [0.0] * n_part
    cx = (0, 1, 1, 0, -1, -1, -1, 0, 1)
    cy = (0, 0, 1, 1, 1, 0, -1, -1, -1)
    nx, ny = int(x_max / (2.0 * r)), int(y_max / (2.0 * r))
    if nx < 1 or ny < 1:
        raise ValueError("the cell must hold at least one particle diameter per side")
    dx, dy = x_max / nx, y_max / ny
    unstable, it = True, 0
    while unstable:
        if it >= max_iterations:
            raise RuntimeError("random_packing did not settle")
        unstable = False
        grid = [[[] for _ in range(ny)] for _ in range(nx)]
        for l in range(n_part):
            grid[int(px[l] / dx) % nx][int(py[l] / dy) % ny].append(l)
        for i in range(nx):
            for j in range(ny):
                for p in grid[i][j]:
                    for l in range(9):
                        for q in grid[(i + cx[l] + nx) % nx][(j + cy[l] + ny) % ny]:
                            for n in range(9):
                                if p != q and p != 0:
                                    # SeedParticle::add_force
                                    xd = px[p] - (px[q] + cx[n] * x_max)
                                    yd = py[p] - (py[q] + cy[n] * y_max)
                                    d = math.sqrt(xd * xd + yd * yd)
                                    if d <= r + r:
                                        c = max(1.0 - 0.99 * d / (r + r), 0.0)
                                        fx[p] += r / 10.0 * c * xd / d
                                        fy[p] += r / 10.0 * c * yd / d
        for i in range(n_part):   # SeedParticle::clamp_force(0.01)
            if fx[i] * fx[i] + fy[i] * fy[i] > 0.01 * 0.01:
                fn = math.sqrt(fx[i] * fx[i] + fy[i] * fy[i])
                fx[i], fy[i] = 0.01 * fx[i] / fn, 0.01 * fy[i] / fn
        unstable = not all(stable)
        for i in range(n_part):   # SeedParticle::advance
            px[i] += fx[i]
            py[i] += fy[i]
            while px[i] < 0:
                px[i] += x_max
            while py[i] < 0:
                py[i] += y_max
            while px[i] > x_max:
                px[i] -= x_max
            while py[i] > y_max:
                py[i] -= y_max
            stable[i] = not ((fx[i] * fx[i] + fy[i] * fy[i]) / (r * r) >= 1e-9)
            fx[i] = fy[i] = 0.0
        it += 1
    return px, py


def load_obj(fname):
    """obj_file_load (mesh_tools.h:103-152): "v x y z" vertices and "f" faces
    of three or four vertex numbers (1-based, anything after a '/' ignored);
    a quad becomes the triangles (0, 1, 2) and (0, 2, 3). Returns (vertices
    (nv, 3) float64, faces (nf, 3) int32, 0-based)."""
    verts, faces = [], []
    with open(fname) as f:
        for line in f:
            t = line.split()
            if not t:
                continue
            if t[0] == "v":
                verts.append((float(t[1]), float(t[2]), float(t[3])))
            elif t[0] == "f":
                ids = [int(w.split("/")[0]) - 1 for w in t[1:]]
                if len(ids) == 3:
                    faces.append(ids)
                elif len(ids) == 4:
                    faces += [[ids[0], ids[1], ids[2]], [ids[0], ids[2], ids[3]]]
    return np.array(verts, np.float64).reshape(-1, 3), np.array(faces, np.int32).reshape(-1, 3)


class Structure:
    """Structure(script) (structure.cpp, lua_structure.cpp): `script` is a
    callable taking this object; it calls size / default_material / add_* /
    declare_parameter like the reference's Lua structure files."""

    def __init__(self, script: Callable[["Structure"], object]):
        self.script = script
        self.params: Dict[str, float] = {}
        self.finalize()

    def finalize(self):
        """Structure::finalize (structure.cpp:138-221): runs the script again."""
        self.lx = self.ly = self.lz = 0.0
        self.default = 0
        self.periodic = [0, 0, 0]
        self.flips = [0, 0, 0]
        self.meshes: List[tuple] = []
        self.ops: List[A.StructureOp] = []
        self.script(self)

    # the functions a structure script calls (structure.cpp:166-187)
    def size(self, lx, ly, lz):
        """Sets lx, ly, lz at once (the script's globals)."""
        self.lx, self.ly, self.lz = float(lx), float(ly), float(lz)

    def declare_parameter(self, name: str, default: float) -> float:
        """structure_declare_parameter (lua_structure.cpp:616-645)."""
        return self.params.setdefault(name, float(default))

    def parameter(self, name: str, value: float):
        """Structure:parameter (lua_structure.cpp:263-281): records the value;
        the next finalize() uses it."""
        self.params[name] = float(value)

    def default_material(self, index: int):
        self.default = int(index)

    def random_packing(self, x_max, y_max, r, n_part, seed=None):
        """The structure scripts' random_packing (see the module function)."""
        return random_packing(x_max, y_max, r, n_part, seed)

    def loop(self, px, py, pz):
        """Structure::set_loop (structure.cpp:338-348): periodic images."""
        self.periodic = [int(px != 0), int(py != 0), int(pz != 0)]

    def flip(self, fx, fy, fz):
        """Structure::set_flip (structure.cpp:326-336): mirrored axes."""
        self.flips = [int(fx != 0), int(fy != 0), int(fz != 0)]

    def _op(self, kind, mat, *p):
        self.ops.append(A.structure_op(kind, mat, *p))

    def add_block(self, x1, x2, y1, y2, z1, z2, index):
        self._op(A.OP_BLOCK, index, x1, x2, y1, y2, z1, z2)

    def add_layer(self, axis: str, z1, z2, index):
        a = 0 if axis in ("X", "x") else (1 if axis in ("Y", "y") else 2)
        self._op(A.OP_LAYER, index, a, z1, z2)

    def add_sphere(self, x, y, z, r, index):
        self._op(A.OP_SPHERE, index, x, y, z, r)

    def add_cylinder(self, x, y, z, dx, dy, dz, r, index):
        # lua_structure.cpp:376-397: from (x, y, z) along (dx, dy, dz)
        self._op(A.OP_CYLINDER, index, x, y, z, x + dx, y + dy, z + dz, r)

    def add_cone(self, x, y, z, dx, dy, dz, r, index):
        """Base centre (x, y, z), apex at (x+dx, y+dy, z+dz), base radius r
        (structure_add_cone)."""
        self._op(A.OP_CONE, index, x, y, z, x + dx, y + dy, z + dz, r)

    def add_ellipsoid(self, x, y, z, rx, ry, rz, index):
        self._op(A.OP_ELLIPSOID, index, x, y, z, rx, ry, rz)

    def add_sin_layer(self, z1, a1, z2, a2, px, phi_x, py, phi_y, index):
        """Layer between z1 + a1 t and z2 + a2 t, t = (sin 2pi(x/px + phi_x)
        + sin 2pi(y/py + phi_y)) / 2 (a period of 0 drops its term)."""
        self._op(A.OP_SIN_LAYER, index, z1, a1, z2, a2, px, phi_x, py, phi_y)

    def add_vect_block(self, xO, yO, zO, xA, yA, zA, xB, yB, zB, xC, yC, zC, index):
        """Parallelepiped at O spanned by the edges A, B, C."""
        self._op(A.OP_VECT_BLOCK, index, xO, yO, zO, xA, yA, zA, xB, yB, zB, xC, yC, zC)

    def add_vect_tri(self, xO, yO, zO, xA, yA, zA, xB, yB, zB, xC, yC, zC, alp, index):
        """Prism at O over the edges A, B, C, slanted by alp along C."""
        self._op(A.OP_VECT_TRI, index, xO, yO, zO, xA, yA, zA, xB, yB, zB, xC, yC, zC, alp)

    def add_coating(self, theta, phi, thickness, delta, origin_index, index):
        """Coats, with material `index`, the cells of `origin_index` that lie
        within `thickness` along the direction (theta, phi) (degrees) above a
        different material, and see only `origin_index` up to the top."""
        self._op(A.OP_COATING, index, theta, phi, thickness, delta, origin_index)

    def add_mesh(self, x, y, z, scale, fname, index):
        """Closed triangle mesh from an OBJ file, vertices multiplied by
        `scale` (structure_add_mesh; the reference records x, y, z but does
        not move the mesh)."""
        self.meshes.append(load_obj(fname))
        self._op(A.OP_MESH, index, x, y, z, scale, len(self.meshes) - 1)

    def add_conformal_coating(self, thickness, delta, origin_index, index):
        """Coats, with material `index`, the cells of `origin_index` closer
        than `thickness` to its surface, sampled every `delta` (0: 5 nm)."""
        self._op(A.OP_CONF_COATING, index, thickness, delta, origin_index)

    def retrieve_nominal_size(self):
        return self.lx, self.ly, self.lz

    def discretize(self, nx, ny, nz, dx, dy, dz, device=0) -> np.ndarray:
        """Structure::discretize on the GPU (aefdtd_discretize): (nz, ny, nx) map."""
        lib = load()
        out = np.zeros(nx * ny * nz, np.uint32)
        arr = (A.StructureOp * max(1, len(self.ops)))(*self.ops)
        desc = A.structure_desc(self.default, self.periodic, self.flips, (self.lx, self.ly, self.lz), self.meshes)
        check(lib.aefdtd_discretize(None, nx, ny, nz, dx, dy, dz, arr, len(self.ops), C.byref(desc),
                                    out.ctypes.data_as(C.POINTER(C.c_uint32)), device), None)
        return out.reshape(nz, ny, nx)


# ---- sensors and sources ------------------------------------------------------

def _orientation(s: str) -> int:
    """is_x_pos / is_x_neg ... (string_tools.cpp:253-300)."""
    for axis, pos, neg in (("x", A.NORMAL_X, A.NORMAL_XM), ("y", A.NORMAL_Y, A.NORMAL_YM),
                           ("z", A.NORMAL_Z, A.NORMAL_ZM)):
        if s.lower() in (axis, "+" + axis, axis + "+"):
            return pos
        if s.lower() in ("-" + axis, axis + "-"):
            return neg
    return -1


def _face(s: str) -> int:
    o = _orientation(s)
    return {A.NORMAL_XM: 0, A.NORMAL_X: 1, A.NORMAL_YM: 2, A.NORMAL_Y: 3, A.NORMAL_ZM: 4, A.NORMAL_Z: 5}.get(o, -1)


class _Located:
    """Location handling shared by Sensor_generator and Source_generator
    (sensors.cpp:142-161, sources.cpp:84-103): real coordinates become cells
    with nearest_integer, and an empty range becomes one cell wide."""

    def __init__(self):
        self.real = (0.0,) * 6
        self.grid = [0] * 6
        self.orient = A.NORMAL_Z

    def location(self, *v):
        """location(x, y, z) or location(x1, x2, y1, y2, z1, z2), in metres."""
        if len(v) == 3:
            v = self._point_real(v)
        self.real = tuple(float(t) for t in v)
        self._is_real = True

    def location_grid(self, *v):
        """location_grid(i, j, k) or location_grid(i1, i2, j1, j2, k1, k2), in cells."""
        g = list(self.grid)
        if len(v) == 3:
            g[0], g[2], g[4] = (int(t) for t in v)
            self._point_grid(g)
        else:
            g = [int(t) for t in v]
        self.grid = g
        self._is_real = False

    _is_real = True

    def orientation(self, s: str):
        o = _orientation(s)
        if o >= 0:
            self.orient = o

    def to_discrete(self, dx, dy, dz):
        if not self._is_real:
            return tuple(self.grid)
        b = [nearest_integer(r / d) for r, d in zip(self.real, (dx, dx, dy, dy, dz, dz))]
        for a in range(3):
            if b[2 * a + 1] <= b[2 * a]:
                b[2 * a + 1] = b[2 * a] + 1
        return tuple(b)


class SensorGen(_Located):
    """create_sensor(type) (lua_sensors.cpp:26-147) for the sensor types of
    this path; defaults of Sensor_generator::Sensor_generator
    (sensors.cpp:27-44)."""

    KINDS = ("planar_spectral_poynting", "box_spectral_poynting", "fieldmap", "fieldmap2", "fieldblock",
             "fieldpoint")

    def __init__(self, kind: str):
        super().__init__()
        if kind not in self.KINDS:
            raise ValueError(f"sensor type {kind!r} is not on this path (available: {', '.join(self.KINDS)})")
        self.kind = kind
        self._name = "sensor"
        self.lmin, self.lmax, self.nl = 470e-9, 850e-9, 481
        self.disabled = 0

    def _point_real(self, v):
        # sensor_set_location_real with 3 arguments sets x1, y1, z1 only
        r = list(self.real)
        r[0], r[2], r[4] = v
        return r

    def _point_grid(self, g):
        pass

    def spectrum(self, lmin, lmax, nl):
        self.lmin, self.lmax, self.nl = float(lmin), float(lmax), int(nl)

    def wavelength(self, lam):
        self.lmin = self.lmax = float(lam)
        self.nl = 1

    def name(self, s: str):
        self._name = s

    def disable(self, face: str):
        f = _face(face)
        if f >= 0:
            self.disabled |= 1 << f


class SourceGen(_Located):
    """create_source("oscillator") (lua_sources.cpp:26-140; defaults of
    sources.cpp:28-42)."""

    def __init__(self, kind: str):
        super().__init__()
        if kind != "oscillator":
            raise ValueError(f"source type {kind!r} is not on this path (available: oscillator)")
        self.kind = kind
        self.lmin, self.lmax = 370e-9, 850e-9

    def _point_real(self, v):
        x, y, z = v
        return (x, x, y, y, z, z)

    def _point_grid(self, g):
        g[1], g[3], g[5] = g[0] + 1, g[2] + 1, g[4] + 1

    def spectrum(self, lmin, lmax):
        self.lmin, self.lmax = float(lmin), float(lmax)


def create_sensor(kind: str) -> SensorGen:
    return SensorGen(kind)


def create_source(kind: str) -> SourceGen:
    return SourceGen(kind)


_rng = {"seed": int(time.time())}


def rng_seed(i: int):
    """rng_seed(i) (base.cpp:68-73): seeds the draws of the FT-mode
    completion probes (the reference's global std::mt19937, seeded from the
    clock by default)."""
    _rng["seed"] = int(i)


# ---- modes ------------------------------------------------------------------

class Mode:
    """MODE(name) for "fdtd_normal", "fdtd" and "fdtd_oblique_ARS" with the
    FDTD_Mode defaults (lua_fd.cpp:40-68, lua_fdtd.cpp:24-42)."""

    NAMES = {"fdtd_normal": A.MODE_NORMAL, "fdtd": A.MODE_CUSTOM, "fdtd_oblique_ARS": A.MODE_OBLIQUE}

    def __init__(self, name: str, precision=A.FP64, device=0):
        if name not in self.NAMES:
            raise ValueError(f"mode {name!r} is not on this path (available: {', '.join(self.NAMES)})")
        self.mode = self.NAMES[name]
        self.precision, self.device = precision, device
        self._struct: Optional[Structure] = None
        self.D = [5e-9, 5e-9, 5e-9]
        self.pad = [0] * 6
        self.pml = [0] * 6
        self.kappa, self.sigma, self.alpha = [25.0] * 6, [1.0] * 6, [0.2] * 6
        self.pol = 0
        self.Nt, self.Ntap, self.tmod = 5000, 0, 1.0
        self.lmin, self.lmax, self.Nl = 370e-9, 850e-9, 481
        self.mats: Dict[int, Material] = {}
        self.sensors: List[SensorGen] = []
        self.sources: List[SourceGen] = []
        self.cc = None                       # ("energy", step, coeff) or ("ft", step, lmin, lmax, coeff, quant, layout)
        self.kp = ("target", {"lmin": 500e-9, "amin_deg": 0.0})
        self.phi = 0.0
        self._prefix = ""

    # discretisation (lua_fd.cpp)
    def Dx(self, d): self.D[0] = float(d)
    def Dy(self, d): self.D[1] = float(d)
    def Dz(self, d): self.D[2] = float(d)
    def Dxyz(self, d): self.D = [float(d)] * 3

    def structure(self, s: Structure):
        """FD_Mode::set_structure (lua_fd.cpp:465-469): evaluates the script
        with the parameters set so far."""
        self._struct = s
        s.finalize()

    def _discretization(self):
        lx, ly, lz = self._struct.retrieve_nominal_size()
        return [max(1, nearest_integer(l / d)) for l, d in zip((lx, ly, lz), self.D)]

    def Nx(self): return self._discretization()[0]
    def Ny(self): return self._discretization()[1]
    def Nz(self): return self._discretization()[2]
    def Lx(self): return self.Nx() * self.D[0]
    def Ly(self): return self.Ny() * self.D[1]
    def Lz(self): return self.Nz() * self.D[2]

    def padding(self, xm, xp, ym, yp, zm, zp): self.pad = [int(v) for v in (xm, xp, ym, yp, zm, zp)]

    def _pml(self, f, n, kappa, sigma, alpha):
        self.pml[f], self.kappa[f], self.sigma[f], self.alpha[f] = int(n), float(kappa), float(sigma), float(alpha)

    def pml_xm(self, n, k, s, a): self._pml(0, n, k, s, a)
    def pml_xp(self, n, k, s, a): self._pml(1, n, k, s, a)
    def pml_ym(self, n, k, s, a): self._pml(2, n, k, s, a)
    def pml_yp(self, n, k, s, a): self._pml(3, n, k, s, a)
    def pml_zm(self, n, k, s, a): self._pml(4, n, k, s, a)
    def pml_zp(self, n, k, s, a): self._pml(5, n, k, s, a)

    def polarization(self, p):
        """FD_mode_set_polarization (lua_fd.cpp:619-645): "TE" / "TM" in any
        case; a number is an angle ("mix"), which both drivers run as TE
        (normal_incidence.cpp:237-238, oblique_biphase.cpp:137)."""
        self.pol = 1 if isinstance(p, str) and p.lower() == "tm" else 0

    def N_tsteps(self, n):
        """Fixed step count; cancels auto_tsteps (FDTD_Mode::set_N_tsteps)."""
        self.Nt = int(n)
        self.cc = None
    def tapering(self, n): self.Ntap = int(n)
    def time_mod(self, m): self.tmod = float(m)
    def prefix(self, s): self._prefix = s
    def output_directory(self, s): pass
    def display_step(self, n): pass

    def spectrum(self, lmin, lmax, nl=None):
        self.lmin, self.lmax = float(lmin), float(lmax)
        if nl is not None:
            self.Nl = int(nl)

    def material(self, index: int, mat):
        """FD_mode_set_material (lua_fd.cpp:576-604): a Material, or the path
        of a material file (located from the working directory, then from the
        directories in `self.search_path`, like locate_file)."""
        if isinstance(mat, str):
            m = Material()
            m.load_script(mat, getattr(self, "search_path", ()))
            mat = m
        if not isinstance(mat, Material):
            raise TypeError("material: a Material or the path of a material file")
        self.mats[int(index)] = mat

    def register_sensor(self, s: SensorGen): self.sensors.append(s)
    def register_source(self, s: SourceGen): self.sources.append(s)

    def auto_tsteps(self, nt, step, *args):
        """(Nt, step, coeff): energy mode; (Nt, step, lmin, lmax, coeff, quant[, layout]): FT mode."""
        self.Nt = int(nt)
        if len(args) == 1:
            self.cc = ("energy", int(step), float(args[0]))
        else:
            lmin, lmax, coeff, quant = args[:4]
            layout = args[4] if len(args) > 4 else "nnb"
            self.cc = ("ft", int(step), float(lmin), float(lmax), float(coeff), int(quant), layout)

    # oblique wavevector sweeps (lua_fdtd.cpp:554-634)
    def kp_auto(self, amin, amax): self.kp = ("auto", {"amin_deg": amin, "amax_deg": amax})
    def kp_full(self, n, kp_ic, kp_fc): self.kp = ("full", {"nkp": n, "kp_ic": kp_ic, "kp_fc": kp_fc})
    def kp_fixed_angle(self, n, lmin, lmax, ang):
        self.kp = ("fixed_angle", {"nkp": n, "lmin": lmin, "lmax": lmax, "amin_deg": ang})
    def kp_fixed_lambda(self, n, lam, amin, amax):
        self.kp = ("fixed_lambda", {"nkp": n, "lmin": lam, "amin_deg": amin, "amax_deg": amax})
    def kp_target(self, lam, ang): self.kp = ("target", {"lmin": lam, "amin_deg": ang})
    def incident_plane(self, phi_deg): self.phi = float(phi_deg)

    # FDTD_Mode::finalize (lua_fdtd.cpp:74-203)
    def _finalize(self, n):
        pml, pad = list(self.pml), list(self.pad)
        if self.mode in (A.MODE_NORMAL, A.MODE_OBLIQUE):
            pml[0:4] = [0, 0, 0, 0]
            pml[4] = pml[4] if pml[4] > 0 else 25
            pml[5] = pml[5] if pml[5] > 0 else 25
        boxes = [(s.to_discrete(*self.D), False) for s in self.sensors]
        boxes += [(s.to_discrete(*self.D), True) for s in self.sources]
        for a in range(3):
            if n[a] <= 1:
                continue
            for side in range(2):
                f = 2 * a + side
                if not pml[f]:
                    pad[f] = 0
                    continue
                p = max(pad[f], 5)
                for b, osc in boxes:
                    margin = 50 if osc else 5
                    p = max(p, margin - b[2 * a]) if side == 0 else max(p, margin + b[2 * a + 1] - n[a])
                pad[f] = p
        return pml, pad

    def scene(self) -> Scene:
        """The grid, map, materials, excitation and sensors compute() runs."""
        if self._struct is None:
            raise ValueError("no structure set")
        n = self._discretization()
        pml, pad = self._finalize(n)
        g = A.grid_desc(n[0], n[1], n[2], self.D[0], self.D[1], self.D[2], mode=self.mode,
                        precision=self.precision, nt=self.Nt, tapering=self.Ntap, time_mod=self.tmod, pml=pml,
                        pad=pad, kappa=self.kappa, sigma=self.sigma, alpha=self.alpha, device=self.device)
        m = self._struct.discretize(n[0], n[1], n[2], *self.D, device=self.device)
        top = int(m.max()) if m.size else 0
        mats = [self.mats.get(i, Material()).desc() for i in range(max(top + 1, max(self.mats, default=0) + 1))]
        planar = [s for s in self.sensors if s.kind in ("planar_spectral_poynting", "fieldmap2")]
        sens = [A.SensorDesc(s.orient, s.to_discrete(*self.D), s.nl, s.lmin, s.lmax) for s in planar]
        # the normal-incidence driver drives its own plane wave and ignores
        # registered sources (normal_incidence.cpp:161-266)
        srcs = ([] if self.mode == A.MODE_NORMAL else
                [A.SourceDesc(s.orient, s.to_discrete(*self.D), s.lmin, s.lmax) for s in self.sources])
        normal = A.NormalDesc(self.pol, self.Nl, self.lmin, self.lmax) if self.mode == A.MODE_NORMAL else None
        obl = (A.ObliqueDesc(self.pol, self.Nl, self.lmin, self.lmax, 0.0, 0.0)
               if self.mode == A.MODE_OBLIQUE else None)
        return Scene(g, m, mats, self.Nt, normal=normal, oblique=obl, sensors=sens, sources=srcs,
                     name=self._prefix or "mode")

    def compute(self) -> dict:
        """Runs the mode's driver; returns its results (see the module text)."""
        sc = self.scene()
        if self.mode == A.MODE_OBLIQUE:
            kind, kw = self.kp
            kw = dict(kw)
            if kind in ("auto", "full"):
                kw.update(lambda_min=self.lmin, lambda_max=self.lmax)
            kps = OBL.kp_list(kind, **kw)
            # several wavevectors advance together as one batch (same results as one by one)
            return {"kp": kps, "obl": OBL.sweep(sc, kps, phi_deg=self.phi, batch=len(kps) > 1)}
        out: dict = {}
        with fdtd.build_simulation(sc) as sim:
            ids = self._add_extra_sensors(sim)
            if self.cc is not None and self.cc[0] == "energy":
                sim.set_completion(self.cc[2], self.cc[1])
            elif self.cc is not None:
                _, step, lmin, lmax, coeff, quant, layout = self.cc
                sim.set_completion_ft(lmin, lmax, coeff, quant, layout, _rng["seed"], step)
            sim.step(self.Nt)
            sim.synchronize()
            out["steps"] = sim.dims().step
            if self.cc is not None:
                out["completion"] = sim.completion()
            if self.mode == A.MODE_NORMAL:
                out["spectra"] = sim.normal_spectra()
            res = []
            for s in self.sensors:
                kind, hid = ids[id(s)]
                if kind == "flux":
                    r = sim.sensor_flux(hid)
                elif kind == "dft":
                    r = sim.sensor_dft(hid)
                elif kind == "box":
                    r = sim.box_flux(hid)
                else:
                    r = sim.fieldmap(hid)
                res.append((s._name, r))
            out["sensors"] = res
        return out

    def _add_extra_sensors(self, sim):
        """Ids of every registered sensor: planar ones were created with the
        scene (in order), the others are added here."""
        ids, planar = {}, 0
        for s in self.sensors:
            b = s.to_discrete(*self.D)
            if s.kind in ("planar_spectral_poynting", "fieldmap2"):
                ids[id(s)] = ("flux" if s.kind == "planar_spectral_poynting" else "dft", planar)
                planar += 1
            elif s.kind == "box_spectral_poynting":
                ids[id(s)] = ("box", sim.add_box_sensor(b, s.nl, s.lmin, s.lmax, s.disabled))
            elif s.kind == "fieldmap":
                ids[id(s)] = ("map", sim.add_fieldmap(A.MAP_PLANE, b, s.lmin, s.orient))
            elif s.kind == "fieldblock":
                ids[id(s)] = ("map", sim.add_fieldmap(A.MAP_BLOCK, b, s.lmin))
            else:
                ids[id(s)] = ("map", sim.add_fieldmap(A.MAP_POINT, b, s.lmin))
        return ids


def MODE(name: str, precision=A.FP64, device=0) -> Mode:
    """MODE(name) (lua_fdtd.cpp, the mode constructor); precision FP32 runs
    the single-precision kernels."""
    return Mode(name, precision, device)
