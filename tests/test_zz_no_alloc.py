"""aefdtd_plane_sums_static: per-plane field sums with no device allocation.

Called through the C ABI on a simulation's own field arrays, on the
simulation's stream, twice in a row (with more steps in between), and checked
against the transmission-plane sums the stepping path reports through
aefdtd_get_plane_sums (slots 9..11 at plane zs_s) and against FP64 sums of the
fields read back with aefdtd_get_field. Tolerance: the plane-sum tolerance of
the parity tests (relative 1e-12 of the summed magnitudes; only the summation
order may differ). This file sorts last so that it also runs after every other
test has used the device; it passes alone in a fresh process too.

Free device memory is recorded before the first call as well (after the
output buffers are made and torch has run its own first kernel): the first
call on a device may load the library's device code there (module data, a few
KiB to MiB, taken once per process), so that growth is bounded; the second
call must leave free memory unchanged.

A tapered step checks the weight path: inside the taper window the stepping
path weights each plane sum by s_curve (mathUT.cpp:1186-1193); the static
call given the same weight must equal slots 9..11 bit for bit."""
import ctypes as C

import numpy as np
import pytest

import scenes
from aether_b200 import _abi as A
from aether_b200 import _lib
from aether_b200 import fdtd

pytestmark = pytest.mark.gpu

RTOL_PLANE = 1e-12
MAX_PLANES = 64


def _out(n):
    """A device output buffer filled with NaN (allocated and written by torch
    before any measurement, so that torch's own first kernel launch and its
    allocator are not counted against the entry point)."""
    import torch

    out = torch.full((n, 3), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    return out


def _static_sums(sim, planes, precision, weight=1.0, out=None):
    lib = _lib.load()
    d = sim.dims()
    ptrs = (C.c_void_p * 3)()
    for c in range(3):
        p = C.c_void_p()
        _lib.check(lib.aefdtd_field_device_ptr(sim._h, c, C.byref(p)))
        ptrs[c] = p.value
    if out is None:
        out = _out(len(planes))
    pl = (C.c_int32 * len(planes))(*planes)
    err = C.create_string_buffer(256)
    st = lib.aefdtd_plane_sums_static(ptrs, precision, d.nx, d.ny, d.nz, pl, len(planes), weight,
                                      C.c_void_p(out.data_ptr()), C.c_void_p(sim.stream_ptr()), err, 256)
    assert st == 0, err.value.decode()
    sim.synchronize()
    return out.cpu().numpy()


def _check(sim, planes, got):
    d = sim.dims()
    ps = sim.plane_sums()
    want = ps[9:12, -1]
    scale = np.abs(want) + 1e-300
    assert np.all(np.abs(got[0] - want) <= RTOL_PLANE * np.maximum(scale, np.abs(got[0]))), (got[0], want)
    for c in range(3):
        f = sim.field(c)
        for i, k in enumerate(planes):
            ref = f[k].sum()
            mag = np.abs(f[k]).sum()
            assert abs(got[i, c] - ref) <= RTOL_PLANE * mag + 1e-300, (c, k, got[i, c], ref)
    assert d.zs_s == planes[0]


@pytest.mark.parametrize("precision", [A.FP64, A.FP32])
def test_static_plane_sums_match_stepping_path_twice(precision):
    import torch

    scene = scenes.slab_tm(precision=precision, nsteps=300)
    assert 77 < scene.grid.nt - scene.grid.tapering  # taper weight 1 at every step used below
    with fdtd.build_simulation(scene) as sim:
        d = sim.dims()
        planes = [d.zs_s, 0, d.zs_s + 3, d.zs_e - 1, d.nz - 1]
        sim.step(40)
        outs = [_out(len(planes)), _out(len(planes))]
        sim.synchronize()
        free_first = torch.cuda.mem_get_info()[0]
        first = _static_sums(sim, planes, precision, out=outs[0])
        assert free_first - torch.cuda.mem_get_info()[0] <= 16 << 20   # module load at most
        _check(sim, planes, first)
        assert np.any(first != 0)
        sim.step(37)
        sim.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        second = _static_sums(sim, planes, precision, out=outs[1])
        free_after = torch.cuda.mem_get_info()[0]
        _check(sim, planes, second)
        assert not np.array_equal(first, second)
        assert free_after == free_before


def test_static_plane_sums_reject_sizes_beyond_scratch():
    lib = _lib.load()
    ptrs = (C.c_void_p * 3)(1, 1, 1)
    planes = (C.c_int32 * (MAX_PLANES + 1))(*([0] * (MAX_PLANES + 1)))
    err = C.create_string_buffer(256)
    st = lib.aefdtd_plane_sums_static(ptrs, A.FP64, 8, 8, 8, planes, MAX_PLANES + 1, 1.0, None, None, err, 256)
    assert st == 1 and b"1 to 64 planes" in err.value
    planes[0] = 8
    st = lib.aefdtd_plane_sums_static(ptrs, A.FP64, 8, 8, 8, planes, 1, 1.0, None, None, err, 256)
    assert st == 1 and b"outside" in err.value


def _s_curve(x, xmin, xmax):
    u = (x - xmin) / (xmax - xmin)
    return 0.0 if u <= 0 else (1.0 if u >= 1.0 else u * u * (3.0 - 2.0 * u))


@pytest.mark.parametrize("precision", [A.FP64, A.FP32])
def test_static_plane_sums_tapered_weight_bit_identical(precision):
    scene = scenes.slab_tm(precision=precision, nsteps=300)
    scene.grid.tapering = 100
    nt, ntap = scene.grid.nt, scene.grid.tapering
    with fdtd.build_simulation(scene) as sim:
        d = sim.dims()
        sim.step(250)
        t = 249                                   # the last step's index
        w = _s_curve(float(t), nt - 1.0, float(nt - ntap))
        assert 0.0 < w < 1.0
        got = _static_sums(sim, [d.zs_s], precision, weight=w)
        want = sim.plane_sums()[9:12, t]
        assert np.any(want != 0)
        assert np.array_equal(got[0], want), (got[0], want)
