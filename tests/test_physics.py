"""Physics checks that need no reference: vacuum transparency and the
analytic Fabry-Perot reflectance of a dielectric slab at normal incidence
(the slab of the 64x64x128 workload, reduced to a thin periodic column since
normal incidence on a laterally uniform slab does not depend on the
transverse size). Run on the CPU oracle and on the GPU FP32 path."""
import numpy as np
import pytest

import oracle_lib
from aether_b200 import _abi as A
from aether_b200 import configs as CF


def fp_reflectance(lam, n, d):
    r12 = (1 - n) / (1 + n)
    delta = 2 * np.pi * n * d / lam
    e = np.exp(2j * delta)
    r = r12 * (1 - e) / (1 - r12 ** 2 * e)
    return np.abs(r)


def slab(n_slab, precision=A.FP64, nsteps=5000):
    return CF.slab_scene(nx=2, ny=2, nz_total=260, pml=16, slab=20, n_slab=n_slab, nsteps=nsteps, nl=31,
                         sensor_gap=10, precision=precision)


def check_fp(spec, n):
    lam = spec[:, 0]
    r = spec[:, 1]
    ana = fp_reflectance(lam, n, 20 * 5e-9)
    assert np.max(np.abs(r - ana)) < 0.02, np.c_[lam, r, ana]


def test_vacuum_is_transparent():
    r = oracle_lib.run(slab(1.0, nsteps=3000), "port", want_fields=False)
    spec = r["spectra"]
    assert np.max(spec[:, 1]) < 5e-3          # |r|
    assert np.max(np.abs(spec[:, 2] - 1)) < 5e-3   # |t|


def test_slab_matches_fabry_perot():
    r = oracle_lib.run(slab(1.5), "port", want_fields=False)
    check_fp(r["spectra"], 1.5)


@pytest.mark.gpu
def test_gpu_fp32_slab_matches_fabry_perot():
    from aether_b200 import fdtd
    r = fdtd.run(slab(1.5, precision=A.FP32), want_fields=False)
    check_fp(r["spectra"], 1.5)
