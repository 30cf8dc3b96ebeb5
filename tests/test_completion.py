"""Energy-mode completion sensor (aefdtd_set_completion) against the
reference's own CompletionSensor, run through the compiled reference core.

The stop step must be the reference's; fields at the stop are bit-identical
(FP64); the spectra, computed over Nt = t steps as the driver does after a
completion, agree to the parity tolerance of the plane-sum spectra."""
import numpy as np
import pytest

import oracle_lib
import scenes
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu

RTOL_SPECTRA = 1e-10


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("every", [40, 64])
def test_completion_stops_where_the_reference_stops(every):
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built")
    sc = scenes.slab_tm(nsteps=3000)
    coeff = 2e-2
    ref = oracle_lib.run_ref_completion(sc, coeff, every, nsteps=3000)
    assert ref["stop"] > 0, "the reference run must complete inside the step limit"
    with fdtd.build_simulation(sc) as s:
        s.set_completion(coeff, every)
        s.step(3000)
        done, stop, ratio = s.completion()
        assert done and stop == ref["stop"]
        assert s.dims().step == stop + 1
        assert np.array_equal(s.fields(), ref["fields"])
        assert abs(ratio - ref["energy_last"] / ref["energy_max"]) <= 1e-12 * abs(ratio)
        assert rel(s.normal_spectra()[:, 1:], ref["spectra"][:, 1:]) < RTOL_SPECTRA
        s.step(100)                      # completed: no further steps
        assert s.dims().step == stop + 1


def test_completion_off_runs_all_steps_and_reset_rearms():
    sc = scenes.slab_tm(nsteps=3000)
    with fdtd.build_simulation(sc) as s:
        s.set_completion(2e-2, 50)
        s.step(3000)
        done, stop, _ = s.completion()
        assert done and stop < 2999 and stop % 50 == 0
        s.reset()
        assert s.completion()[0] is False
        s.set_completion(0.0, 50)       # off
        s.step(3000)
        assert s.dims().step == 3000 and s.completion()[0] is False
