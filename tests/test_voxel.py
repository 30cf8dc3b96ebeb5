"""Cell tagging (Structure::discretize): the oracle restatement against
independent numpy tagging on the CPU, and the device voxeliser against the
oracle bit-for-bit on the GPU, including corners that sit exactly on
primitive boundaries."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib
from aether_b200 import _abi as A

_P = C.POINTER


def oracle_vox(nx, ny, nz, d, ops, default=0, periodic=(0, 0, 0), lengths=(0, 0, 0)):
    lib = C.CDLL(oracle_lib.PORT_PATH)
    fn = lib.aeoracle_voxelize
    fn.argtypes = [C.c_int32] * 3 + [C.c_double] * 3 + [_P(A.StructureOp), C.c_int32, C.c_int32,
                                                      _P(C.c_int32), _P(C.c_double), _P(C.c_uint32)]
    out = np.zeros(nx * ny * nz, np.uint32)
    arr = (A.StructureOp * max(len(ops), 1))(*ops)
    per = (C.c_int32 * 3)(*periodic)
    ln = (C.c_double * 3)(*lengths)
    fn(nx, ny, nz, d[0], d[1], d[2], arr, len(ops), default, per, ln, out.ctypes.data_as(_P(C.c_uint32)))
    return out.reshape(nz, ny, nx)


def op(kind, mat, *p):
    o = A.StructureOp()
    o.kind, o.mat_index = kind, mat
    for i, v in enumerate(p):
        o.p[i] = v
    return o


def random_ops(rng, L, n=12, nmat=5):
    ops = []
    for _ in range(n):
        k = rng.integers(0, 4)
        m = int(rng.integers(1, nmat))
        if k == A.OP_BLOCK:
            a = rng.uniform(0, L, 3)
            b = rng.uniform(0, L, 3)
            ops.append(op(k, m, a[0], b[0], a[1], b[1], a[2], b[2]))
        elif k == A.OP_LAYER:
            z = np.sort(rng.uniform(0, L, 2))
            ops.append(op(k, m, float(rng.integers(0, 3)), z[0], z[1]))
        elif k == A.OP_SPHERE:
            c = rng.uniform(0, L, 3)
            ops.append(op(k, m, c[0], c[1], c[2], rng.uniform(0.05, 0.4) * L))
        else:
            a = rng.uniform(0, L, 3)
            b = rng.uniform(0, L, 3)
            ops.append(op(k, m, a[0], a[1], a[2], b[0], b[1], b[2], rng.uniform(0.05, 0.2) * L))
    return ops


def test_oracle_sphere_and_block_match_numpy():
    d = 5e-9
    nx, ny, nz = 21, 19, 23
    ops = [op(A.OP_BLOCK, 1, 2 * d, 10 * d, 0, 7 * d, 3 * d, 3 * d + 1e-12),
           op(A.OP_SPHERE, 2, 10 * d, 9 * d, 11 * d, 6 * d)]
    m = oracle_vox(nx, ny, nz, (d, d, d), ops)
    i = np.arange(nx) * d
    j = np.arange(ny) * d
    k = np.arange(nz) * d
    Z, Y, X = np.meshgrid(k, j, i, indexing="ij")
    ref = np.zeros((nz, ny, nx), np.uint32)
    blk = (X >= 2 * d) & (X < 10 * d) & (Y >= 0) & (Y < 7 * d) & (Z >= 3 * d) & (Z < 3 * d + 1e-12)
    ref[blk] = 1
    dx, dy, dz = X - 10 * d, Y - 9 * d, Z - 11 * d
    sph = dx * dx + dy * dy + dz * dz <= (6 * d) * (6 * d)
    ref[sph] = 2
    assert np.array_equal(m, ref)
    assert (m == 2).sum() > 0 and (m == 1).sum() > 0


def test_oracle_last_operation_wins_and_default():
    d = 1e-9
    ops = [op(A.OP_LAYER, 3, 2.0, 0, 5e-9), op(A.OP_LAYER, 4, 2.0, 2e-9, 3e-9)]
    m = oracle_vox(4, 4, 8, (d, d, d), ops, default=7)
    assert list(m[:, 0, 0]) == [3, 3, 4, 3, 3, 7, 7, 7]


def test_oracle_periodic_images():
    d = 1e-9
    L = 10e-9
    ops = [op(A.OP_SPHERE, 1, 0.0, 5e-9, 5e-9, 2.5e-9)]
    m = oracle_vox(10, 10, 10, (d, d, d), ops, periodic=(1, 0, 0), lengths=(L, L, L))
    # a sphere centred on x=0 shows up at both x edges through the periodic image
    assert m[5, 5, 0] == 1 and m[5, 5, 9] == 1 and m[5, 5, 5] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_gpu_voxelize_bit_identical_to_oracle(seed):
    from aether_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(seed)
    d = (2.5e-9, 3e-9, 2e-9)
    nx, ny, nz = 37, 29, 41
    L = 80e-9
    ops = random_ops(rng, L)
    # a sphere whose surface passes exactly through grid corners
    ops.append(op(A.OP_SPHERE, 9, 10 * d[0], 10 * d[1], 10 * d[2], 5 * d[0]))
    periodic = (seed % 2, 0, 1 if seed == 2 else 0)
    lengths = (nx * d[0], ny * d[1], nz * d[2])
    ref = oracle_vox(nx, ny, nz, d, ops, default=0, periodic=periodic, lengths=lengths)
    out = np.zeros(nx * ny * nz, np.uint32)
    arr = (A.StructureOp * len(ops))(*ops)
    st = lib.aefdtd_voxelize(None, nx, ny, nz, d[0], d[1], d[2], arr, len(ops), 0,
                             (C.c_int32 * 3)(*periodic), (C.c_double * 3)(*lengths),
                             out.ctypes.data_as(_P(C.c_uint32)), 0)
    assert st == 0
    assert np.array_equal(out.reshape(nz, ny, nx), ref)
