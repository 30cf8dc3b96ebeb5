"""Pins the CPU restatement (oracle/fdtd_oracle.cpp) to the reference.

1. Against the committed golden fixtures, which were produced by the
   reference's own FDTD core compiled from source (tests/golden/make_golden.py):
   bit-exact fields (SHA-256), plane sums, R/T spectra and flux spectra.
2. Where oracle/_ref was built here, against the reference core directly on
   further seeded scenes, also bit-exact."""
import hashlib
import os

import numpy as np
import pytest

import oracle_lib
import scenes

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
GOLDEN = ["slab_tm", "slab_te", "gold_sphere", "debye_lorentz_sphere", "custom_box", "thin_column"]


def sha(fields):
    f = np.ascontiguousarray(fields, dtype=np.float64)
    return [hashlib.sha256(f[c].tobytes()).hexdigest() for c in range(6)]


@pytest.mark.parametrize("name", GOLDEN)
def test_port_matches_reference_golden(name):
    g = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    r = oracle_lib.run(scenes.ALL[name](), "port")
    assert np.array_equal(r["dims"], g["dims"])
    assert sha(r["fields"]) == list(g["field_sha256"])
    if "fields" in g:
        assert np.array_equal(r["fields"], g["fields"])
    if "plane_sums" in g:
        assert np.array_equal(r["plane_sums"], g["plane_sums"])
        assert np.array_equal(r["spectra"], g["spectra"])
    for i, f in enumerate(r["flux"]):
        assert np.array_equal(f, g[f"flux{i}"])


needs_ref = pytest.mark.skipif(not oracle_lib.available("ref"), reason="oracle/_ref not built here")


@needs_ref
@pytest.mark.parametrize("seed", [1, 2])
def test_port_matches_reference_random_custom(seed):
    sc = scenes.custom_box(nsteps=60, seed=100 + seed, n_dielectric=4 + seed)
    a = oracle_lib.run(sc, "ref")
    b = oracle_lib.run(sc, "port")
    assert np.array_equal(a["fields"], b["fields"])
    for fa, fb in zip(a["flux"], b["flux"]):
        assert np.array_equal(fa, fb)


@needs_ref
def test_port_matches_reference_many_materials():
    sc = scenes.custom_many_materials(nsteps=40)
    assert sc.map.max() > 255
    a = oracle_lib.run(sc, "ref")
    b = oracle_lib.run(sc, "port")
    assert np.array_equal(a["fields"], b["fields"])


@needs_ref
def test_port_matches_reference_tapering():
    from aether_b200 import _abi as A
    sc = scenes.slab_tm(nsteps=80)
    sc.grid.nt = 80
    sc.grid.tapering = 30
    a = oracle_lib.run(sc, "ref")
    b = oracle_lib.run(sc, "port")
    assert np.array_equal(a["plane_sums"], b["plane_sums"])
    assert np.array_equal(a["spectra"], b["spectra"])
    for fa, fb in zip(a["flux"], b["flux"]):
        assert np.array_equal(fa, fb)
