"""Algorithmic byte counts of the stepping kernels (the roofline numerator)
and the Gcell-updates/s metric.

Fused time step (one pass per step, leapfrog.cuh): per interior cell-update
12*s + b_id bytes -- the six old field values read once, the six new ones
written once, the material id read once. CPML and dispersive add-ons as below.

Split half-steps:
Per interior cell-update the E and H half-steps together move 18*s + b_id
bytes (s = 8 for FP64, 4 for FP32; b_id = 1 or 2): each kernel reads its own
3 components and the other family's 3 components once and writes its 3
components, assuming perfect neighbour reuse, and the E kernel reads the
material id. Add-ons: per CPML axis a cell lies in, the E (H) kernel
read-modify-writes two psi arrays (+4*s each side); a dispersive cell with
Np poles read-modify-writes 3*Np complex psi values in the E kernel
(+12*Np*s)."""
from __future__ import annotations

import numpy as np

from . import _abi as A


def cell_counts(scene):
    """Counts cells in each CPML range and dispersive cells of the total grid."""
    nx, ny, nz = scene.total_dims()
    pml, pad = scene.padded_faces()
    g = scene.grid

    def ranges(n, pm, pp, e_side):
        idx = np.arange(n)
        if not (pm or pp):
            return np.zeros(n, bool)
        if e_side:
            return ((idx >= 1) & (idx < pm)) | (idx >= n - pp + 1)
        return (idx < pm) | ((idx >= n - pp) & (idx < n - 1))

    out = {"cells": nx * ny * nz}
    for side in ("E", "H"):
        e = side == "E"
        rx = ranges(nx, pml[0], pml[1], e).sum() * ny * nz
        ry = ranges(ny, pml[2], pml[3], e).sum() * nx * nz
        rz = ranges(nz, pml[4], pml[5], e).sum() * nx * ny
        out[f"pml_{side}"] = int(rx + ry + rz)
    # dispersive cells: structure map cells (pads replicate edge slices)
    poles = np.zeros(len(scene.materials), np.int64)
    for i, m in enumerate(scene.materials):
        poles[i] = m.n_debye + m.n_drude + m.n_lorentz + m.n_critpoint
    # plane by plane over the total grid (no full-size temporaries)
    nx_, ny_, nz_ = scene.total_dims()
    xs, ys, zs = pml[0] + pad[0], pml[2] + pad[2], pml[4] + pad[4]
    m = scene.map
    xi = np.clip(np.arange(nx_) - xs, 0, m.shape[2] - 1)
    yi = np.clip(np.arange(ny_) - ys, 0, m.shape[1] - 1)
    counts = np.zeros(len(poles), np.int64)
    for k in range(nz_):
        plane = m[min(max(k - zs, 0), m.shape[0] - 1)][np.ix_(yi, xi)]
        counts += np.bincount(np.minimum(plane.ravel(), len(poles) - 1), minlength=len(poles))[:len(poles)]
    out["disp_pole_cells"] = int((counts * poles).sum())
    out["id_bytes"] = 1 if int(m.max()) < 256 else 2
    return out


def expand_map(scene):
    """Total-grid material map with pad/PML replication (FDTD::set_matsgrid)."""
    nx, ny, nz = scene.total_dims()
    pml, pad = scene.padded_faces()
    xs, ys, zs = pml[0] + pad[0], pml[2] + pad[2], pml[4] + pad[4]
    m = scene.map
    xi = np.clip(np.arange(nx) - xs, 0, m.shape[2] - 1)
    yi = np.clip(np.arange(ny) - ys, 0, m.shape[1] - 1)
    zi = np.clip(np.arange(nz) - zs, 0, m.shape[0] - 1)
    return m[np.ix_(zi, yi, xi)]


def kernel_bytes(scene, precision=None):
    """Algorithmic bytes per launch of the E and H half-step kernels."""
    s = 8 if (scene.grid.precision if precision is None else precision) == A.FP64 else 4
    c = cell_counts(scene)
    e = c["cells"] * (9 * s + c["id_bytes"]) + c["pml_E"] * 4 * s + c["disp_pole_cells"] * 12 * s
    h = c["cells"] * 9 * s + c["pml_H"] * 4 * s
    return {"E": int(e), "H": int(h), "cells": c["cells"], "detail": c, "elem_bytes": s}


def fused_bytes(scene, precision=None):
    """Algorithmic bytes of one fused time step over the whole grid."""
    s = 8 if (scene.grid.precision if precision is None else precision) == A.FP64 else 4
    c = cell_counts(scene)
    return int(c["cells"] * (12 * s + c["id_bytes"]) + (c["pml_E"] + c["pml_H"]) * 4 * s
               + c["disp_pole_cells"] * 12 * s)


def gcells(cells, steps, seconds):
    return cells * steps / seconds / 1e9


def step_bytes(scene, precision=None, dft_block=64, fused=False):
    """Algorithmic bytes of one whole time step: the E and H half-steps (or
    the fused step), the sensor samples (per point: 18 field reads, 6 sample
    writes) and, per step, 1/K of each DFT block (samples read once, FP64
    complex accumulators read and written for every wavelength)."""
    kb = kernel_bytes(scene, precision)
    s = kb["elem_bytes"]
    total = fused_bytes(scene, precision) if fused else kb["E"] + kb["H"]
    for sd in scene.sensors:
        x1, x2, y1, y2, z1, z2 = sd.box
        span = [max(1, x2 - x1), max(1, y2 - y1), max(1, z2 - z1)]
        span.sort()
        P = span[1] * span[2]
        total += P * (18 + 6) * s
        total += (P * 6 * s * dft_block + 2 * 6 * sd.nl * P * 16) / dft_block
    return int(total)
