"""The oblique driver's wavevector lists (aether_b200.oblique.kp_list, a
restatement of FDTD_oblique_biphase_get_kp, oblique_biphase.cpp:503-597):
host logic only."""
import math

import pytest

from aether_b200 import oblique

NM = 1e-9


def test_auto_is_geometric_from_lambda_max():
    kps = oblique.kp_list("auto", lambda_min=400 * NM, lambda_max=1000 * NM, amin_deg=10, amax_deg=60)
    r = math.sin(math.radians(60)) / math.sin(math.radians(10))
    assert kps[0] == pytest.approx(2 * math.pi / (1000 * NM) * math.sin(math.radians(60)), rel=1e-15)
    for a, b in zip(kps, kps[1:]):
        assert b / a == pytest.approx(r, rel=1e-12)
    # count: lambda_n = lambda_max (sin amin / sin amax)^n, stop once <= lambda_min
    n, lam = 1, 1000 * NM / r
    while lam > 400 * NM:
        lam /= r
        n += 1
    assert len(kps) == n


def test_full_clamps_and_spans():
    kps = oblique.kp_list("full", lambda_min=400 * NM, lambda_max=1000 * NM, nkp=5, kp_ic=-1.0, kp_fc=2.0)
    assert len(kps) == 5 and kps[0] == 0.0          # kp_ic clamped to 0: zero angle
    m_c = 0.99 * math.pi / 2 * 0.95                  # kp_fc clamped to 0.95
    lam = 400 * NM + math.cos(m_c) * 600 * NM
    assert kps[-1] == pytest.approx(2 * math.pi / lam * math.sin(math.pi / 2 * math.sin(m_c)), rel=1e-14)
    assert oblique.kp_list("full", lambda_min=400 * NM, lambda_max=1000 * NM, nkp=1)[0] > 0   # Nkp 1: m_ct = 1


def test_fixed_angle_fixed_lambda_and_target():
    fa = oblique.kp_list("fixed_angle", nkp=3, lmin=500 * NM, lmax=900 * NM, amin_deg=30)
    assert fa[0] == pytest.approx(2 * math.pi / (900 * NM) * 0.5, rel=1e-14)
    assert fa[-1] == pytest.approx(2 * math.pi / (500 * NM) * 0.5, rel=1e-14)
    fl = oblique.kp_list("fixed_lambda", nkp=4, lmin=600 * NM, amin_deg=0, amax_deg=60)
    assert fl[0] == 0.0 and fl[-1] == pytest.approx(2 * math.pi / (600 * NM) * math.sin(math.radians(60)), rel=1e-14)
    t = oblique.kp_list("target", lmin=700 * NM, amin_deg=45)
    assert t == [pytest.approx(2 * math.pi / (700 * NM) * math.sin(math.radians(45)), rel=1e-15)]
    with pytest.raises(ValueError):
        oblique.kp_list("bogus")
