"""The x/y-CPML group's y-only items on the two-cells-per-thread kernel
(e_pmly_v2 / h_pmly_v2): tiles in a y-CPML range or on a y PEC plane with no
x-CPML cell take the pair kernel with the y (and z) psi recursions; tiles with
x-CPML cells keep the one-cell kernel.

FP64: fields and flux bit-identical to the one-cell kernel for the same items
(AEFDTD_PAIR without the x/y-CPML bit) on custom-mode scenes with CPML on all
six faces: pairs, lone 32-column tiles, the y = 0 and y = Ny - 1 PEC rows, a
width that leaves a partial last tile, 16-bit material ids; the pair kernel
is launched (more launches per step) and covers the same cells. FP32: within
1e-5 relative (contraction may differ)."""
import hashlib
import os

import numpy as np
import pytest

from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu

NO_PY = {A.FP64: "2", A.FP32: "3"}   # the default pair groups without the x/y-CPML bit


def sha(f):
    f = np.ascontiguousarray(f, dtype=np.float64)
    return [hashlib.sha256(f[c].tobytes()).hexdigest() for c in range(f.shape[0])]


def run(scene, pairs_py, steps):
    env = {"AEFDTD_FUSED": "0", "AEFDTD_TMA": "0"}
    if not pairs_py:
        env["AEFDTD_PAIR"] = NO_PY[scene.grid.precision]
    saved = {k: os.environ.get(k) for k in list(env) + ["AEFDTD_PAIR"]}
    os.environ.pop("AEFDTD_PAIR", None)
    os.environ.update(env)
    try:
        with fdtd.build_simulation(scene) as s:
            s.enable_timing(True, mode=2)   # direct launches: the launch count shows the kernels
            s.step(steps)
            s.synchronize()
            return {"fields": s.fields(), "flux": [s.sensor_flux(i) for i in range(len(scene.sensors))],
                    "launches": s.launch_count(), "groups": s.group_timings(), "dims": s.dims()}
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


SCENES = {
    # pairs (x 64..127), a lone tile beside the x-CPML tile (x 32..63), a partial last tile
    "pml6_150": lambda p: CF.random_spheres_scene(n_total=(150, 40, 48), pml=8, n_dielectric=10, n_lorentz=3,
                                                  r_range=(8e-9, 20e-9), nsteps=80, nl=5, precision=p, seed=11),
    # wider y-CPML slabs than the tile height, dispersive spheres crossing them
    "pml6_wide": lambda p: CF.random_spheres_scene(n_total=(200, 72, 40), pml=12, n_dielectric=20, n_lorentz=4,
                                                   r_range=(6e-9, 18e-9), nsteps=70, nl=5, precision=p, seed=21),
    # 16-bit material ids
    "pml6_ids16": lambda p: CF.random_spheres_scene(n_total=(200, 48, 40), pml=6, n_dielectric=300, n_lorentz=2,
                                                    r_range=(3e-9, 8e-9), nsteps=60, nl=5, precision=p, seed=3),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_pmly_pairs_fp64_bit_identical(name):
    sc = SCENES[name](A.FP64)
    a = run(sc, True, sc.nsteps)
    b = run(sc, False, sc.nsteps)
    assert sha(a["fields"]) == sha(b["fields"])
    assert np.count_nonzero(b["fields"]) > 0
    for x, y in zip(a["flux"], b["flux"]):
        assert np.array_equal(x, y)
    # the pair kernel ran: one more launch per half-step, the same cells per group
    assert a["launches"] > b["launches"]
    d = a["dims"]
    for h in "EH":
        ca = sum(c for (hh, _), (_, c) in a["groups"].items() if hh == h)
        assert ca == d.nx * d.ny * d.nz
        assert a["groups"][(h, "pml_xy")][1] == b["groups"][(h, "pml_xy")][1]


def test_pmly_pairs_fp32_close():
    sc = SCENES["pml6_wide"](A.FP32)
    a = run(sc, True, sc.nsteps)
    b = run(sc, False, sc.nsteps)
    d = np.linalg.norm(a["fields"] - b["fields"]) / np.linalg.norm(b["fields"])
    assert d < 1e-5, d
    assert a["launches"] > b["launches"]
