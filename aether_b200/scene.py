"""Plain description of one FDTD run: the arguments a mode driver hands to the
core (grid, structure map, materials, excitation, sensors, step count).

The reference builds the same objects from a Lua script: FDTD_Mode::finalize
(src/finite_differences/FDTD/modes/lua_fdtd.cpp:74-203) sizes pads and PML,
Structure::discretize gives the map, and the driver functions create the FDTD,
Material, sensor and source objects (normal_incidence.cpp:161-266,
default_fdtd.cpp:24-98)."""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

from . import _abi as A

C_LIGHT = 299792458.0


@dataclasses.dataclass
class Scene:
    grid: A.GridDesc
    map: np.ndarray                       # (nz, ny, nx) uint32 structure map
    materials: List[A.MaterialDesc]
    nsteps: int
    normal: Optional[A.NormalDesc] = None
    oblique: Optional[A.ObliqueDesc] = None   # mode OBLIQUE: polarization, spectrum, in-plane k
    sensors: List[A.SensorDesc] = dataclasses.field(default_factory=list)
    sources: List[A.SourceDesc] = dataclasses.field(default_factory=list)
    name: str = "scene"

    def __post_init__(self):
        self.map = np.ascontiguousarray(self.map, dtype=np.uint32)
        g = self.grid
        if self.map.shape != (g.nz, g.ny, g.nx):
            raise ValueError(f"map shape {self.map.shape} != (nz, ny, nx)=({g.nz},{g.ny},{g.nx})")

    # ---- geometry of the total grid (FDTD constructor, fdtd_core.cpp:158-251)
    def padded_faces(self):
        g = self.grid
        pml = list(g.pml)
        pad = list(g.pad)
        if g.mode in (A.MODE_NORMAL, A.MODE_OBLIQUE):
            pml[:4] = [0, 0, 0, 0]
            pad[:4] = [0, 0, 0, 0]
            pad[4] = max(5, pad[4])
            pad[5] = max(5, pad[5])
        else:
            for ax in range(3):
                if pml[2 * ax] or pml[2 * ax + 1]:
                    pad[2 * ax] = max(5, pad[2 * ax])
                    pad[2 * ax + 1] = max(5, pad[2 * ax + 1])
        return pml, pad

    def total_dims(self):
        g = self.grid
        pml, pad = self.padded_faces()
        nx = g.nx + pml[0] + pad[0] + pad[1] + pml[1]
        ny = g.ny + pml[2] + pad[2] + pad[3] + pml[3]
        nz = g.nz + pml[4] + pad[4] + pad[5] + pml[5]
        return nx, ny, nz

    @property
    def cells(self) -> int:
        nx, ny, nz = self.total_dims()
        return nx * ny * nz

    def dt(self) -> float:
        g = self.grid
        if g.dt > 0:
            return g.dt
        return min(min(g.dx, g.dy), g.dz) / (math.sqrt(3.0) * C_LIGHT) * 0.99 * g.time_mod

    def flux_lengths(self):
        return [s.nl for s in self.sensors]
