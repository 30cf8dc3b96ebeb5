"""Oblique incidence (mode OBLIQUE, aefdtd_setup_oblique) against the
reference's own oblique driver run in the compiled reference core
(FDTD_oblique_biphase_comp with two OBL_PHASE grids and Bloch_Wideband).

FP64: both grids' fields within relative L2 1e-12 and the per-step R/T sums
within 1e-11 of their largest magnitude. The only deviation from the
reference's arithmetic is the incident field's 30001-line sums, whose sines
and cosines come from the device's sincos instead of the host's cexp (a few
ulp per term). Spectra (ratios of DFTs of those sums) within 1e-8 absolute on
|r|, |t| and 1e-8 on the phases where the amplitude is above 1e-6. FP32:
fields within relative L2 1e-3 of the FP64 reference, |r| and |t| within
1e-3."""
import numpy as np
import pytest

import oracle_lib
from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def need_ref():
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built")


CASES = {
    "te_kx": dict(kx_in=0.4, ky_in=0.0, polarization=0),
    "tm_kxky_disk": dict(kx_in=0.3, ky_in=0.25, polarization=1),
    "te_normal": dict(kx_in=0.0, ky_in=0.0, polarization=0, disk=False),
    "tm_ky_nodisk": dict(kx_in=0.0, ky_in=0.5, polarization=1, disk=False),
}


@pytest.mark.parametrize("case", list(CASES))
def test_fp64_fields_series_spectra_match_reference(case):
    need_ref()
    steps = 400
    sc = CF.oblique_scene(nsteps=steps, **CASES[case])
    ref = oracle_lib.run_ref_oblique(sc, nsteps=steps)
    got = fdtd.run(sc, nsteps=steps)
    assert np.array_equal(got["dims"], ref["dims"])
    assert np.any(ref["fields"] != 0) and np.any(ref["fields_imag"] != 0)
    assert rel(got["fields"], ref["fields"]) < 1e-12
    assert rel(got["fields_imag"], ref["fields_imag"]) < 1e-12
    s_ref, s_got = ref["series"], got["plane_sums"]
    assert np.max(np.abs(s_got - s_ref)) <= 1e-11 * np.max(np.abs(s_ref))
    sp_ref, sp_got = ref["spectra"], got["spectra"]
    assert sp_got.shape == sp_ref.shape
    assert np.array_equal(sp_got[:, 0], sp_ref[:, 0])
    assert np.max(np.abs(sp_got[:, 1] - sp_ref[:, 1])) < 1e-9
    for a in (2, 4, 6, 8):
        assert np.max(np.abs(sp_got[:, a] - sp_ref[:, a])) < 1e-8 * max(1.0, np.max(np.abs(sp_ref[:, a])))
        big = sp_ref[:, a] > 1e-6
        d = np.angle(np.exp(1j * (sp_got[big, a + 1] - sp_ref[big, a + 1])))
        assert np.all(np.abs(d) < 1e-8)


def test_fp32_close_to_fp64_reference():
    need_ref()
    steps = 400
    sc = CF.oblique_scene(nsteps=steps, **CASES["tm_kxky_disk"])
    ref = oracle_lib.run_ref_oblique(sc, nsteps=steps)
    got = fdtd.run(CF.oblique_scene(nsteps=steps, precision=A.FP32, **CASES["tm_kxky_disk"]), nsteps=steps)
    assert rel(got["fields"], ref["fields"]) < 1e-3
    assert rel(got["fields_imag"], ref["fields_imag"]) < 1e-3
    for a in (2, 4, 6, 8):
        assert np.max(np.abs(got["spectra"][:, a] - ref["spectra"][:, a])) < 1e-3


def test_graphs_pieces_and_reset_agree(monkeypatch):
    """Captured segments against direct launches in uneven pieces, and a
    reset run against a fresh one: bit-identical (FP64)."""
    sc = CF.oblique_scene(nsteps=200, **CASES["tm_kxky_disk"])
    a = fdtd.run(sc, nsteps=200)
    monkeypatch.setenv("AEFDTD_NO_GRAPHS", "1")
    with fdtd.build_simulation(sc) as s:
        for n in (1, 63, 70, 66):
            s.step(n)
        assert np.array_equal(s.fields(), a["fields"])
        assert np.array_equal(s.fields(1), a["fields_imag"])
        assert np.array_equal(s.oblique_series(), a["plane_sums"])
        s.reset()
        s.step(200)
        assert np.array_equal(s.fields(1), a["fields_imag"])


def test_setup_checks():
    sc = CF.oblique_scene(nsteps=10)
    with fdtd.Simulation(sc.grid) as s:
        s.set_material_map(sc.map)
        for i, m in enumerate(sc.materials):
            s.set_material(i, m)
        with pytest.raises(Exception):
            s.step(1)                                   # needs aefdtd_setup_oblique
        with pytest.raises(Exception):
            s.setup_normal(A.NormalDesc(0, 5, 400e-9, 800e-9))   # wrong mode
        s.setup_oblique(sc.oblique)
        with pytest.raises(Exception):
            s.setup_oblique(sc.oblique)                 # once
        s.step(3)
        assert s.oblique_series().shape == (3, 18)


def test_kp_sweep_runs_each_wavevector():
    """aether_b200.oblique.sweep: one run per kp at the incident-plane angle,
    each equal to the single run at that kx, ky."""
    from aether_b200 import oblique
    import math
    sc = CF.oblique_scene(nsteps=150, disk=False)
    kps = oblique.kp_list("fixed_lambda", nkp=2, lmin=700e-9, amin_deg=10, amax_deg=30)
    res = oblique.sweep(sc, kps, phi_deg=30, nsteps=150)
    assert len(res) == 2
    for kp, r in zip(kps, res):
        sc1 = CF.oblique_scene(nsteps=150, disk=False)
        phi = 30 * (math.pi / 180.0)
        sc1.oblique.kx_in, sc1.oblique.ky_in = kp * math.cos(phi), kp * math.sin(phi)
        assert np.array_equal(fdtd.run(sc1, nsteps=150)["spectra"], r)


def test_kp_sweep_in_one_batch_matches_sequential_runs():
    """The oblique driver's wavevector sweep advanced as one batch (each
    wavevector a subset of its own) gives the sequential runs' spectra and
    R/T sums bit for bit (FP64)."""
    from aether_b200 import oblique as OBL
    from aether_b200 import configs as CF
    sc = CF.oblique_scene(nsteps=300)
    kps = OBL.kp_list("fixed_lambda", nkp=3, lmin=600e-9, amin_deg=10, amax_deg=40)
    seq = OBL.sweep(sc, kps, phi_deg=20)
    bat = OBL.sweep(sc, kps, phi_deg=20, batch=True)
    for a, b in zip(seq, bat):
        assert np.array_equal(a, b)


def test_kp_sweep_in_chunks_matches_sequential_runs():
    """A sweep with more wavevectors than one batch holds (capped at two per
    batch here; by the device's memory otherwise) runs them batch after batch
    and still gives the sequential spectra bit for bit (FP64)."""
    from aether_b200 import oblique as OBL
    from aether_b200 import configs as CF
    sc = CF.oblique_scene(nsteps=200)
    kps = OBL.kp_list("fixed_lambda", nkp=5, lmin=600e-9, amin_deg=5, amax_deg=45)
    seq = OBL.sweep(sc, kps, phi_deg=10)
    bat = OBL.sweep(sc, kps, phi_deg=10, batch=True, max_chunk=2)
    assert len(bat) == len(kps)
    for a, b in zip(seq, bat):
        assert np.array_equal(a, b)
    free, total = fdtd.device_memory(0)
    assert 0 < free <= total
