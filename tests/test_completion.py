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


# FT mode. The reference draws its probes from its global generator; the
# driver reseeds it (seedp) before creating the sensor, so both sides draw the
# same cells and wavelengths. Layouts whose per-face rounding leaves probes
# unassigned are avoided: the reference leaves those probes' cells
# uninitialised (CompletionSensor::initialize, s_completion.cpp:286-358) and
# reads past its grids with them.
@pytest.mark.parametrize("coeff,layout,npts,seed", [(2e-2, "nnb", 40, 7), (1e-2, "v", 30, 3),
                                                   (5e-2, "bnn", 24, 11)])
def test_ft_completion_stops_where_the_reference_stops(coeff, layout, npts, seed):
    if not oracle_lib.available("ref"):
        pytest.skip("reference core not built")
    sc = scenes.slab_tm(nsteps=6000)
    ref = oracle_lib.run_ref_completion_ft(sc, 400e-9, 1000e-9, coeff, npts, layout, seed, 50, nsteps=6000)
    assert ref["stop"] > 0, "the reference run must complete inside the step limit"
    with fdtd.build_simulation(sc) as s:
        s.set_completion_ft(400e-9, 1000e-9, coeff, npts, layout, seed, 50)
        s.step(6000)
        done, stop, open_ratio = s.completion()
        assert done and stop == ref["stop"]
        assert open_ratio <= 0.1
        assert np.array_equal(s.fields(), ref["fields"])
        assert rel(s.normal_spectra()[:, 1:], ref["spectra"][:, 1:]) < RTOL_SPECTRA


def test_ft_completion_replaced_by_energy_mode_and_reset():
    sc = scenes.slab_tm(nsteps=6000)
    with fdtd.build_simulation(sc) as s:
        s.set_completion_ft(400e-9, 1000e-9, 2e-2, 40, "nnb", 7, 50)
        s.step(6000)
        stop_ft = s.completion()[1]
        s.reset()
        assert s.completion()[0] is False
        s.step(6000)
        assert s.completion()[1] == stop_ft          # the same probes after a reset
        s.reset()
        s.set_completion(2e-2, 50)                    # energy mode replaces FT mode
        s.step(3000)
        assert s.completion()[0] and s.completion()[2] < 2e-2
