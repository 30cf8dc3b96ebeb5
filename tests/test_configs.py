"""The benchmark workloads at full size.

The slab (64x64x128 at 5 nm, n = 1.5 slab, 16-cell CPML on z, 4000 steps, 61
wavelengths, flux planes above and below): the FP64 GPU path against the
reference core compiled from source, fields bit-identical, spectra and flux
to 1e-10 relative. The CPML grading is the reference's (order 4); grading
order 3 is the grid descriptor's pml_m, outside what the reference can run.

The slab and the 128x128x256 dispersive unit cell (gold sphere, 20000 steps, 201
wavelengths): the FP32 path's R/T spectra against the FP64 path (itself
bit-identical to the reference on every golden scene) within 1e-4 absolute,
flux within 1e-3 relative. The measured errors are printed."""
import hashlib

import numpy as np
import pytest

import oracle_lib
from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu

FP32_ABS_RT = 1e-4
FP32_REL_FLUX = 1e-3


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_slab_fp64_full_size_matches_reference():
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built")
    sc = CF.slab_scene(precision=A.FP64)
    ref = oracle_lib.run(sc, "ref")
    got = fdtd.run(sc)
    assert [sha(f) for f in got["fields"]] == [sha(f) for f in ref["fields"]]
    assert rel(got["spectra"][:, 1:], ref["spectra"][:, 1:]) < 1e-10
    for a, b in zip(got["flux"], ref["flux"]):
        assert rel(a, b) < 1e-10


def rt_error(scene_fn):
    r64 = fdtd.run(scene_fn(A.FP64), want_fields=False)
    r32 = fdtd.run(scene_fn(A.FP32), want_fields=False)
    d = np.abs(r32["spectra"][:, 1:3] - r64["spectra"][:, 1:3]).max()
    fl = max(rel(a, b) for a, b in zip(r32["flux"], r64["flux"]))
    return d, fl


@pytest.mark.parametrize("name", ["slab", "gold_sphere"])
def test_fp32_rt_error_against_fp64(name):
    if name == "slab":
        fn = lambda p: CF.slab_scene(precision=p)
    else:
        fn = lambda p: CF.sphere_scene(nx=128, ny=128, nz_total=256, dx=2.5e-9, pml=24, radius=40e-9,
                                       nsteps=20000, nl=201, precision=p)
    d, fl = rt_error(fn)
    print(f"{name}: FP32 max |d r|,|d t| = {d:.3e}, flux rel L2 = {fl:.3e}")
    assert d < FP32_ABS_RT
    assert fl < FP32_REL_FLUX
