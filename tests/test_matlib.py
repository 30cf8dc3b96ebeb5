"""Material files (the reference's mat_lib/*.lua) through aether_b200.matlib.

CPU: the subset reader on small scripts (arithmetic and its precedence,
comments, strings, lists, the loader's calls, a run-time error stopping the
script as lua_pcall does, constructs outside the subset); every file of the
reference's library loaded or refused as recorded in tests/golden/mat_lib.json
(regenerated from the tree when it is present). GPU: scenes using the
recorded terms of two library files (Vial's gold, Drude + 2 critical points;
Rakic's gold, Drude + 5 Lorentz terms), FP64, fields bit-identical to the
reference core given the same terms."""
import glob
import hashlib
import json
import math
import os

import numpy as np
import pytest

import oracle_lib
import scenes
from aether_b200 import _abi as A
from aether_b200 import configs as CF
from aether_b200 import fdtd
from aether_b200 import lua_api as L
from aether_b200 import matlib

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "mat_lib.json")
REFERENCE = os.environ.get("AEFDTD_REFERENCE", os.path.join(os.sep, "root", "reference"))


def script(tmp_path, text, name="m.lua"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_arithmetic_comments_strings(tmp_path):
    m = matlib.load_file(script(tmp_path, """
-- a comment
--[[ a block
     comment ]]
description('line one\\nline two')
name("Test " .. 2 .. " x")
ih=1.0/6.58211951440e-16
wp=9.03; C1=wp/(0.415)
epsilon_infty(2^-1 + -2^2 * 3 - 7 % 3)
add_drude(math.sqrt(0.760)*wp*ih,0.053*ih)
add_lorentz(0.024*C1*C1,0.415*ih,0.241*ih)
add_crit_point(1, 2, -math.pi, 0x10)
add_debye(79.2,9.4e-12)
validity_range(250e-9,6200e-9)
"""))
    assert m.error is None and m.refusal() is None
    assert m.description == "line one\nline two"
    assert m.name == "Test 2 x"
    assert m.eps_inf == 0.5 + -(2.0 ** 2) * 3 - 1
    ih = 1.0 / 6.58211951440e-16
    assert m.terms["drude"] == [(math.sqrt(0.760) * 9.03 * ih, 0.053 * ih)]
    c1 = 9.03 / 0.415
    assert m.terms["lorentz"] == [(0.024 * c1 * c1, 0.415 * ih, 0.241 * ih)]
    assert m.terms["critpoint"] == [(1.0, 2.0, -math.pi, 16.0)]
    assert m.terms["debye"] == [(79.2, 9.4e-12)]
    assert m.validity == (250e-9, 6200e-9)


def test_runtime_error_stops_the_script_like_pcall(tmp_path):
    m = matlib.load_file(script(tmp_path, "epsilon_infty(3)\nset_constant()\nadd_drude(1, 2)\n"))
    assert m.eps_inf == 3.0 and m.terms["drude"] == []
    assert "set_constant" in m.error and "Lua error" in m.refusal()


def test_models_the_fdtd_cannot_run_are_refused(tmp_path):
    for body, why in (("add_sellmeier(1.0, 0.006)", "Sellmeier"), ("add_cauchy(1.5, 0.01)", "Cauchy"),
                      ("l={4e-7,5e-7}\nnr={1.5,1.6}\nni={0,0}\nadd_data_index(l,nr,ni)", "tabulated"),
                      ("effective_type('bruggeman')", "effective")):
        m = matlib.load_file(script(tmp_path, "epsilon_infty(2)\n" + body + "\n"))
        assert why in m.refusal()
        with pytest.raises(ValueError):
            m.desc()


def test_constructs_outside_the_subset_are_rejected(tmp_path):
    for body in ("for i=1,3 do add_drude(1,1) end", "function f() end", "if x then end", "a = 7 // 2"):
        with pytest.raises(matlib.SubsetError):
            matlib.load_file(script(tmp_path, body))


def test_load_script_and_front_end(tmp_path):
    inner = script(tmp_path, "epsilon_infty(4)\nadd_drude(1e16, 1e14)\n", "inner.lua")
    outer = script(tmp_path, "add_lorentz(1, 2, 3)\nload_script('inner.lua')\n", "outer.lua")
    m = matlib.load_file(outer)
    assert m.eps_inf == 4.0 and m.terms["drude"] == [(1e16, 1e14)] and m.terms["lorentz"] == []   # reset
    mode = L.MODE("fdtd_normal")
    mode.search_path = (str(tmp_path),)
    mode.material(1, "inner.lua")
    d = mode.mats[1].desc()
    assert d.eps_inf == 4.0 and d.n_drude == 1


def test_fixture_covers_every_library_file():
    with open(FIXTURE) as f:
        fx = json.load(f)
    assert len(fx) >= 30
    assert all(v["status"] in ("loaded", "refused") for v in fx.values())
    assert all((v["status"] == "refused") == bool(v["reason"]) for v in fx.values())
    assert fx["Au_400n_1000n_Vial.lua"]["status"] == "loaded"
    assert fx["N-BK7.lua"]["status"] == "refused"
    files = sorted(glob.glob(os.path.join(REFERENCE, "mat_lib", "*.lua")))
    if not files:
        pytest.skip("reference tree absent: fixture checked on its own")
    assert sorted(os.path.basename(p) for p in files) == sorted(fx)
    for p in files:
        m = matlib.load_file(p)
        want = fx[os.path.basename(p)]
        assert m.refusal() == want["reason"], p
        assert m.eps_inf == want["eps_inf"], p
        assert {k: [list(t) for t in v] for k, v in m.terms.items()} == want["terms"], p


def fixture_desc(name):
    with open(FIXTURE) as f:
        v = json.load(f)[name]
    assert v["status"] == "loaded"
    t = v["terms"]
    return A.material_desc(v["eps_inf"], debye=[tuple(x) for x in t["debye"]], drude=[tuple(x) for x in t["drude"]],
                           lorentz=[tuple(x) for x in t["lorentz"]], critpoint=[tuple(x) for x in t["critpoint"]])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["Au_400n_1000n_Vial.lua", "Au_Rakic.lua"])
def test_library_gold_fp64_bit_identical_to_reference(name):
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built")
    sc = CF.sphere_scene(nx=12, ny=10, nz_total=90, dx=2.5e-9, pml=8, radius=8e-9, nsteps=250, nl=7, sensor_gap=4,
                         precision=A.FP64, material=fixture_desc(name))
    ref = oracle_lib.run(sc, "ref")
    got = fdtd.run(sc)

    def sha(f):
        return [hashlib.sha256(np.ascontiguousarray(f[c], np.float64).tobytes()).hexdigest() for c in range(6)]

    assert sha(got["fields"]) == sha(ref["fields"])
    for a, b in zip(got["flux"], ref["flux"]):
        assert np.linalg.norm(a - b) <= 1e-10 * np.linalg.norm(b)
