"""Bounded device waits: a wait that runs out reports AEFDTD_TIMEOUT and
leaves the handle usable.

The FP32 tensor-core DFT waits on an mbarrier for its phasor copies and for
the MMA commit. The test hook aefdtd_test_hook withholds the copies, so the
first wait of every CTA runs out after a short bound (2^20 SM cycles, under a
millisecond). No GPU fault is involved: each CTA sets the handle's error
flag, frees its tensor memory and returns. The next synchronising call must
return AEFDTD_TIMEOUT; after the hook is cleared and the handle reset, a run
must give the same results as a fresh handle (which it cannot if any CTA
kept its tensor memory: the next allocation would not be granted)."""
import numpy as np
import pytest

import scenes
from aether_b200 import _abi as A
from aether_b200 import _lib
from aether_b200 import fdtd
from aether_b200._lib import AefdtdError

pytestmark = pytest.mark.gpu

WAIT_CYCLES, WITHHOLD = 1, 2   # AEFDTD_TEST_DFT_WAIT_CYCLES, AEFDTD_TEST_DFT_WITHHOLD_COPY
TIMEOUT = 3


def test_dft_wait_runs_out_then_handle_recovers():
    sc = scenes.gold_sphere(precision=A.FP32, nsteps=192)
    want = fdtd.run(sc)
    lib = _lib.load()
    with fdtd.build_simulation(sc) as s:
        _lib.check(lib.aefdtd_test_hook(s._h, WAIT_CYCLES, 1 << 20))
        _lib.check(lib.aefdtd_test_hook(s._h, WITHHOLD, 1))
        with pytest.raises(AefdtdError) as e:
            s.step(192)          # two DFT blocks accumulated within the run
            s.synchronize()
        assert e.value.status == TIMEOUT
        # the flag was read and cleared: the handle answers again
        s.synchronize()
        _lib.check(lib.aefdtd_test_hook(s._h, WITHHOLD, 0))
        _lib.check(lib.aefdtd_test_hook(s._h, WAIT_CYCLES, 1 << 32))
        s.reset()
        s.step(192)
        s.synchronize()
        assert np.array_equal(s.fields(), want["fields"])
        for i, f in enumerate(want["flux"]):
            assert np.array_equal(s.sensor_flux(i), f)


def test_hook_rejects_unknown_and_bad_values():
    sc = scenes.gold_sphere(precision=A.FP32, nsteps=64)
    lib = _lib.load()
    with fdtd.build_simulation(sc) as s:
        assert lib.aefdtd_test_hook(s._h, 99, 1) == 1
        assert lib.aefdtd_test_hook(s._h, WAIT_CYCLES, 0) == 1
