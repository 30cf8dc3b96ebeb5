"""Seeded synthetic scenes for the benchmark configurations.

No public dataset is involved: every geometry is generated here from a seed,
with the sizes and parameter distributions of the five workload descriptions
(slab, dispersive sphere, large random grid, metasurface unit cells, serving
mix). Each builder takes size overrides so tests can run the same scene shape
at small scale."""
from __future__ import annotations

import math

import numpy as np

from . import _abi as A
from .scene import Scene

NM = 1e-9


def gold_cp_model():
    """Gold-like Drude + two critical points: eps_inf=1.1, wp=1.3e16 rad/s,
    gamma=1.1e14 rad/s; CP terms A=0.9/1.3, phi=-0.8/-0.5 rad,
    Omega=4.0e15/5.6e15 rad/s, Gamma=1.1e15/1.9e15 rad/s. Parameter order is
    the reference's add_drude(wd, g) and add_crit_point(A, O, P, G)
    (src/materials/lua_material.cpp:122-172)."""
    return A.material_desc(1.1, drude=[(1.3e16, 1.1e14)],
                           critpoint=[(0.9, 4.0e15, -0.8, 1.1e15), (1.3, 5.6e15, -0.5, 1.9e15)])


def lorentz_model():
    """eps_inf=2.0, delta_eps=1.5, w0=3.0e15 rad/s, gamma=1.0e14 rad/s as
    add_lorentz(A, O, G) (dielec_models.cpp:332-358)."""
    return A.material_desc(2.0, lorentz=[(1.5, 3.0e15, 1.0e14)])


def const_n(n):
    return A.material_desc(n * n)


def _normal_grid(nx, ny, nz_s, dx, pml, precision, nt, time_mod=0.5 / 0.99, alpha=0.05):
    return A.grid_desc(nx, ny, nz_s, dx, mode=A.MODE_NORMAL, precision=precision, nt=nt,
                       time_mod=time_mod, pml=(0, 0, 0, 0, pml, pml), pad=(0, 0, 0, 0, 5, 5),
                       kappa=(1.0,) * 6, sigma=(1.0,) * 6, alpha=(alpha,) * 6)


def slab_scene(nx=64, ny=64, nz_total=128, dx=5 * NM, pml=16, slab=20, n_slab=1.5, nsteps=4000,
               nl=61, lmin=400 * NM, lmax=1000 * NM, polarization=1, precision=A.FP64,
               sensor_gap=10):
    """Plain slab: periodic x/y, CPML on +/-z, vacuum with a non-dispersive
    slab of `slab` cells centred in z, x-polarised ("TM") pulse over
    lmin..lmax, Courant 0.5 of the 3-D limit, planar flux sensors above and
    below the slab. nz_total is the total grid height (structure + 2 pads of
    5 + 2 PML)."""
    nz_s = nz_total - 2 * pml - 10
    if nz_s < slab + 2 * sensor_gap + 4:
        raise ValueError("grid too short for the slab and sensors")
    m = np.zeros((nz_s, ny, nx), np.uint32)
    c = (nz_total // 2) - (pml + 5)
    k0 = c - slab // 2
    m[k0:k0 + slab] = 1
    g = _normal_grid(nx, ny, nz_s, dx, pml, precision, nsteps)
    sens = [
        A.SensorDesc(A.NORMAL_ZM, (0, nx, 0, ny, k0 - sensor_gap, k0 - sensor_gap + 1), nl, lmin, lmax),
        A.SensorDesc(A.NORMAL_Z, (0, nx, 0, ny, k0 + slab + sensor_gap, k0 + slab + sensor_gap + 1), nl, lmin, lmax),
    ]
    return Scene(g, m, [const_n(1.0), const_n(n_slab)], nsteps,
                 normal=A.NormalDesc(polarization, nl, lmin, lmax), sensors=sens, name="slab")


def oblique_scene(nx=24, ny=20, nz_total=96, dx=5 * NM, pml=12, kx_in=0.4, ky_in=0.0, slab=10, disk=True,
                  nsteps=600, nl=31, lmin=400 * NM, lmax=1000 * NM, polarization=0, precision=A.FP64):
    """Oblique incidence ("fdtd_oblique_ARS", one in-plane wavevector): a
    periodic cell with a dielectric slab on an n=1.45 substrate, optionally a
    gold-like disk (Drude + critical points) on the slab, CPML on +/-z. kx_in,
    ky_in are fractions of 2 pi / lmax (the driver's k_in, rad/m in vacuum)."""
    nz_s = nz_total - 2 * pml - 10
    m = np.zeros((nz_s, ny, nx), np.uint32)
    sub_top = nz_s // 3
    m[:sub_top] = 2
    m[sub_top:sub_top + slab] = 3
    if disk:
        x = (np.arange(nx) - nx / 2 + 0.5) * dx
        y = (np.arange(ny) - ny / 2 + 0.5) * dx
        r = 0.3 * min(nx, ny) * dx
        inside = (x[None, :] ** 2 + y[:, None] ** 2) <= r * r
        m[sub_top + slab:sub_top + slab + 4][:, inside] = 1
    g = A.grid_desc(nx, ny, nz_s, dx, mode=A.MODE_OBLIQUE, precision=precision, nt=nsteps,
                    time_mod=0.5 / 0.99, pml=(0, 0, 0, 0, pml, pml), pad=(0, 0, 0, 0, 5, 5),
                    kappa=(1.0,) * 6, sigma=(1.0,) * 6, alpha=(0.05,) * 6)
    k0 = 2 * math.pi / lmax
    od = A.ObliqueDesc(polarization, nl, lmin, lmax, kx_in * k0, ky_in * k0)
    return Scene(g, m, [const_n(1.0), gold_cp_model(), const_n(1.45), const_n(1.9)], nsteps, oblique=od,
                 name="oblique")


def sphere_scene(nx=128, ny=128, nz_total=256, dx=2.5 * NM, pml=24, radius=40 * NM, n_sub=1.45,
                 nsteps=20000, nl=201, lmin=400 * NM, lmax=1000 * NM, polarization=1,
                 precision=A.FP64, material=None, sensor_gap=12):
    """Dispersive unit cell: a sphere (gold-like Drude + 2 CP by default)
    resting on an n_sub half-space, periodic x/y, CPML on z, normal
    incidence, planar flux sensors above the sphere and inside the
    substrate."""
    nz_s = nz_total - 2 * pml - 10
    r_cells = radius / dx
    sub_top = int(round(0.3 * nz_s))
    cz = sub_top + r_cells
    if cz + r_cells + sensor_gap + 4 > nz_s:
        raise ValueError("grid too short for the sphere")
    m = np.zeros((nz_s, ny, nx), np.uint32)
    m[:sub_top] = 2
    # cell corners (i*dx, j*dy, k*dz) tested with x^2+y^2+z^2 <= r^2
    # (Add_Sphere::index, structure_primitives.cpp:490-499)
    x = np.arange(nx) * dx - (nx // 2) * dx
    y = np.arange(ny) * dx - (ny // 2) * dx
    z = np.arange(nz_s) * dx - cz * dx
    inside = (z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2) <= radius ** 2
    m[inside] = 1
    g = _normal_grid(nx, ny, nz_s, dx, pml, precision, nsteps)
    top = int(math.ceil(cz + r_cells)) + sensor_gap
    sens = [
        A.SensorDesc(A.NORMAL_Z, (0, nx, 0, ny, top, top + 1), nl, lmin, lmax),
        A.SensorDesc(A.NORMAL_ZM, (0, nx, 0, ny, sub_top - sensor_gap, sub_top - sensor_gap + 1), nl, lmin, lmax),
    ]
    mat = gold_cp_model() if material is None else material
    return Scene(g, m, [const_n(1.0), mat, const_n(n_sub)], nsteps,
                 normal=A.NormalDesc(polarization, nl, lmin, lmax), sensors=sens, name="sphere")


def random_spheres_scene(n_total=(1024, 1024, 512), dx=5 * NM, pml=32, n_dielectric=500,
                         n_lorentz=50, r_range=(20 * NM, 80 * NM), eps_range=(2.0, 12.0),
                         nsteps=5000, seed=1234, precision=A.FP32, lambda0=600 * NM,
                         bandwidth=300 * NM, nl=0):
    """Large single grid in custom mode: CPML on all six faces, seeded random
    non-dispersive spheres (own material index each, eps uniform) plus
    Lorentz spheres sharing one material index, and an Oscillator point source
    at the centre (lambda0 +/- bandwidth/2)."""
    rng = np.random.default_rng(seed)
    pad = 5
    nx_s = n_total[0] - 2 * pml - 2 * pad
    ny_s = n_total[1] - 2 * pml - 2 * pad
    nz_s = n_total[2] - 2 * pml - 2 * pad
    m = np.zeros((nz_s, ny_s, nx_s), np.uint32)
    mats = [const_n(1.0), lorentz_model()]
    x = np.arange(nx_s) * dx
    y = np.arange(ny_s) * dx
    z = np.arange(nz_s) * dx
    L = np.array([nx_s, ny_s, nz_s]) * dx
    specs = []
    for i in range(n_dielectric):
        eps = rng.uniform(*eps_range)
        mats.append(A.material_desc(eps))
        specs.append((len(mats) - 1, rng.uniform(0, 1, 3) * L, rng.uniform(*r_range)))
    for i in range(n_lorentz):
        specs.append((1, rng.uniform(0, 1, 3) * L, rng.uniform(*r_range)))
    for idx, c, r in specs:  # later operations win (Structure::index, structure.cpp:238-255)
        i0, i1 = np.searchsorted(x, c[0] - r), np.searchsorted(x, c[0] + r, side="right")
        j0, j1 = np.searchsorted(y, c[1] - r), np.searchsorted(y, c[1] + r, side="right")
        k0, k1 = np.searchsorted(z, c[2] - r), np.searchsorted(z, c[2] + r, side="right")
        if i0 >= i1 or j0 >= j1 or k0 >= k1:
            continue
        xx = x[i0:i1] - c[0]
        yy = y[j0:j1] - c[1]
        zz = z[k0:k1] - c[2]
        ins = (zz[:, None, None] ** 2 + yy[None, :, None] ** 2 + xx[None, None, :] ** 2) <= r * r
        sub = m[k0:k1, j0:j1, i0:i1]
        sub[ins] = idx
    lmin = lambda0 - bandwidth / 2
    lmax = lambda0 + bandwidth / 2
    g = A.grid_desc(nx_s, ny_s, nz_s, dx, mode=A.MODE_CUSTOM, precision=precision, nt=nsteps,
                    time_mod=0.5 / 0.99, pml=(pml,) * 6, pad=(pad,) * 6,
                    kappa=(1.0,) * 6, sigma=(1.0,) * 6, alpha=(0.05,) * 6)
    cx, cy, cz = nx_s // 2, ny_s // 2, nz_s // 2
    src = A.SourceDesc(A.NORMAL_Z, (cx, cx + 1, cy, cy + 1, cz, cz + 1), lmin, lmax)
    sens = []
    if nl > 0:
        sens.append(A.SensorDesc(A.NORMAL_Z, (0, nx_s, 0, ny_s, nz_s - 2, nz_s - 1), nl, lmin, lmax))
    return Scene(g, m, mats, nsteps, sources=[src], sensors=sens, name="random_spheres")


def metasurface_cell(rng, dx=5 * NM, nz_total=200, pml=16, nsteps=8000, nl=101,
                     lmin=400 * NM, lmax=1000 * NM, precision=A.FP32, period_range=(200 * NM, 600 * NM),
                     flux_planes=True):
    """One nanodisk metasurface unit cell: period ~ U(period_range) (square),
    disk radius ~ U(0.15, 0.45) x period, height ~ U(20, 100) nm, gold-like
    model or dielectric n ~ U(1.8, 3.5) by coin flip, on an n=1.45 substrate."""
    period = rng.uniform(*period_range)
    n = max(8, int(round(period / dx)))
    radius = rng.uniform(0.15, 0.45) * n * dx
    height = rng.uniform(20 * NM, 100 * NM)
    gold = rng.uniform() < 0.5
    n_diel = rng.uniform(1.8, 3.5)
    nz_s = nz_total - 2 * pml - 10
    sub_top = int(round(0.35 * nz_s))
    h_cells = max(1, int(round(height / dx)))
    m = np.zeros((nz_s, n, n), np.uint32)
    m[:sub_top] = 2
    x = (np.arange(n) - n // 2) * dx
    disk = (x[None, :] ** 2 + x[:, None] ** 2) <= radius ** 2
    m[sub_top:sub_top + h_cells][:, disk] = 1
    mat = gold_cp_model() if gold else const_n(n_diel)
    g = _normal_grid(n, n, nz_s, dx, pml, precision, nsteps)
    top = min(nz_s - 3, sub_top + h_cells + 10)
    sens = [A.SensorDesc(A.NORMAL_Z, (0, n, 0, n, top, top + 1), nl, lmin, lmax),
            A.SensorDesc(A.NORMAL_ZM, (0, n, 0, n, max(0, sub_top - 8), max(1, sub_top - 7)), nl, lmin, lmax)]
    if not flux_planes:
        sens = []   # R/T from the normal-mode plane sums only
    return Scene(g, m, [const_n(1.0), mat, const_n(1.45)], nsteps,
                 normal=A.NormalDesc(1, nl, lmin, lmax), sensors=sens, name="metasurface")
