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


@pytest.mark.skipif(not oracle_lib.available("ref"), reason="reference build absent")
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_restatement_matches_reference_structure(seed):
    """The CPU restatement of the four basic primitives against the
    reference's own Structure::discretize (oracle/_ref), periodic images
    included."""
    rng = np.random.default_rng(100 + seed)
    d = (2.5e-9, 3e-9, 2e-9)
    nx, ny, nz = 31, 27, 35
    L = 75e-9
    ops = random_ops(rng, L, n=14)
    ops.append(op(A.OP_SPHERE, 9, 10 * d[0], 10 * d[1], 10 * d[2], 5 * d[0]))
    periodic = (seed % 2, (seed // 2) % 2, 1 if seed == 3 else 0)
    lengths = (nx * d[0], ny * d[1], nz * d[2])
    ref = oracle_lib.ref_discretize(nx, ny, nz, d, ops, A.structure_desc(2, periodic, (0, 0, 0), lengths))
    port = oracle_vox(nx, ny, nz, d, ops, default=2, periodic=periodic, lengths=lengths)
    assert np.array_equal(port, ref)
    assert len(np.unique(ref)) > 3


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



# ---- every primitive of the reference, against its own Structure code ----------

def random_ops_all(rng, L, n=16, nmat=6):
    """Random operations of every kind the device voxeliser has, coatings
    excluded; some sit on grid-aligned coordinates so that corners fall on
    their surfaces."""
    ops = random_ops(rng, L, n=n // 2, nmat=nmat)
    for _ in range(n - n // 2):
        k = int(rng.integers(A.OP_CONE, A.OP_VECT_TRI + 1))
        m = int(rng.integers(1, nmat))
        if k == A.OP_CONE:
            a = rng.uniform(0, L, 3)
            b = rng.uniform(-0.5 * L, 0.5 * L, 3)
            ops.append(op(k, m, a[0], a[1], a[2], a[0] + b[0], a[1] + b[1], a[2] + b[2], rng.uniform(0.05, 0.3) * L))
        elif k == A.OP_ELLIPSOID:
            c = rng.uniform(0, L, 3)
            r = rng.uniform(0.05, 0.4, 3) * L
            ops.append(op(k, m, c[0], c[1], c[2], r[0], r[1], r[2]))
        elif k == A.OP_SIN_LAYER:
            z = np.sort(rng.uniform(0, L, 2))
            px = 0.0 if rng.random() < 0.25 else rng.uniform(0.2, 1.0) * L
            ops.append(op(k, m, z[0], rng.uniform(-0.1, 0.1) * L, z[1], rng.uniform(-0.1, 0.1) * L, px,
                          rng.uniform(0, 1), rng.uniform(0.2, 1.0) * L, rng.uniform(0, 1)))
        else:
            o = rng.uniform(0, 0.6 * L, 3)
            e = rng.uniform(-0.4, 0.4, (3, 3)) * L + np.diag(rng.uniform(0.2, 0.5, 3) * L)
            extra = [rng.uniform(0, 1)] if k == A.OP_VECT_TRI else []
            ops.append(op(k, m, *o, *e[0], *e[1], *e[2], *extra))
    # an axis-aligned vector block on grid corners and a grid-aligned cone axis
    ops.append(op(A.OP_VECT_BLOCK, 7, 0.2 * L, 0.2 * L, 0.2 * L, 0.3 * L, 0, 0, 0, 0.25 * L, 0, 0, 0, 0.2 * L))
    ops.append(op(A.OP_CONE, 8, 0.5 * L, 0.5 * L, 0.1 * L, 0.5 * L, 0.5 * L, 0.6 * L, 0.2 * L))
    rng.shuffle(ops)
    return ops


@pytest.mark.skipif(not oracle_lib.available("ref"), reason="reference build absent")
def test_reference_structure_build_tags_every_primitive():
    rng = np.random.default_rng(5)
    L = 80e-9
    ops = random_ops_all(rng, L, n=20)
    d = (2.5e-9,) * 3
    m = oracle_lib.ref_discretize(32, 32, 32, d, ops, A.structure_desc(0, (1, 1, 0), (0, 1, 0), (L, L, L)))
    kinds = {ops[i].kind for i in range(len(ops))}
    assert {A.OP_CONE, A.OP_ELLIPSOID, A.OP_VECT_BLOCK} <= kinds
    assert len(np.unique(m)) >= 5


def _gpu_discretize(nx, ny, nz, d, ops, desc):
    from aether_b200 import _lib
    lib = _lib.load()
    out = np.zeros(nx * ny * nz, np.uint32)
    arr = (A.StructureOp * max(len(ops), 1))(*ops)
    st = lib.aefdtd_discretize(None, nx, ny, nz, d[0], d[1], d[2], arr, len(ops), C.byref(desc),
                               out.ctypes.data_as(_P(C.c_uint32)), 0)
    _lib.check(st)
    return out.reshape(nz, ny, nx)


@pytest.mark.gpu
@pytest.mark.skipif(not oracle_lib.available("ref"), reason="reference build absent")
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_gpu_every_primitive_bit_identical_to_reference(seed):
    rng = np.random.default_rng(200 + seed)
    L = 90e-9
    d = (2.5e-9, 3e-9, 2e-9)
    nx, ny, nz = 37, 29, 45
    ops = random_ops_all(rng, L, n=24)
    periodic = (seed % 2, (seed // 2) % 2, 0)
    flip = ((seed + 1) % 2, 0, seed // 3)
    desc = A.structure_desc(int(rng.integers(0, 3)), periodic, flip, (nx * d[0], ny * d[1], nz * d[2]))
    ref = oracle_lib.ref_discretize(nx, ny, nz, d, ops, desc)
    gpu = _gpu_discretize(nx, ny, nz, d, ops, desc)
    assert np.array_equal(gpu, ref), np.argwhere(gpu != ref)[:5]
    assert len(np.unique(ref)) >= 5


@pytest.mark.gpu
@pytest.mark.skipif(not oracle_lib.available("ref"), reason="reference build absent")
@pytest.mark.parametrize("case", ["directional", "conformal", "nested", "periodic"])
def test_gpu_coatings_bit_identical_to_reference(case):
    """Add_Coating (a shell grown along a direction over the origin material
    it rests on) and Add_Conf_Coating (a shell of given thickness over the
    origin material's surface), alone, stacked, and with periodic images."""
    L = 60e-9
    d = (2.5e-9,) * 3
    n = 24
    base = [op(A.OP_LAYER, 1, 2.0, 0.0, 20e-9),
            op(A.OP_SPHERE, 1, 30e-9, 30e-9, 20e-9, 12e-9),
            op(A.OP_BLOCK, 2, 5e-9, 20e-9, 35e-9, 55e-9, 15e-9, 32e-9)]
    if case == "directional":
        ops = base + [op(A.OP_COATING, 3, 20.0, 30.0, 6e-9, 1e-9, 0)]
    elif case == "conformal":
        ops = base + [op(A.OP_CONF_COATING, 3, 7.5e-9, 2.5e-9, 0)]
    elif case == "nested":
        ops = base + [op(A.OP_CONF_COATING, 3, 5e-9, 2.5e-9, 0), op(A.OP_COATING, 4, 0.0, 0.0, 4e-9, 1e-9, 0),
                      op(A.OP_CONF_COATING, 5, 4e-9, 0.0, 0)]
    else:
        ops = base + [op(A.OP_SPHERE, 2, 0.0, 30e-9, 25e-9, 10e-9), op(A.OP_CONF_COATING, 3, 6e-9, 3e-9, 0)]
    periodic = (1, 1, 0) if case == "periodic" else (0, 0, 0)
    desc = A.structure_desc(0, periodic, (0, 0, 0), (L, L, L))
    ref = oracle_lib.ref_discretize(n, n, n, d, ops, desc)
    gpu = _gpu_discretize(n, n, n, d, ops, desc)
    assert np.array_equal(gpu, ref), np.argwhere(gpu != ref)[:5]
    assert (ref == 3).sum() > 0


@pytest.mark.gpu
def test_gpu_discretize_rejects_what_the_reference_cannot_finish():
    from aether_b200 import _lib
    desc = A.structure_desc(0, (0, 0, 0), (0, 0, 0), (60e-9,) * 3)
    for bad in ([op(A.OP_COATING, 3, 90.0, 0.0, 5e-9, 1e-9, 0)],          # march through z never ends
                [op(A.OP_COATING, 3, 10.0, 0.0, 5e-9, 0.0, 0)],           # zero step
                [op(A.OP_CONF_COATING, 3 + q, 2e-9, 5e-9, 0) for q in range(4)]):  # nests 4 deep
        with pytest.raises(_lib.AefdtdError):
            _gpu_discretize(8, 8, 8, (5e-9,) * 3, bad, desc)


def icosphere(center, radius, levels=2):
    """Closed triangle mesh of a sphere (subdivided icosahedron)."""
    t = (1 + 5 ** 0.5) / 2
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    v = [np.array(p, float) / np.linalg.norm(p) for p in v]
    for _ in range(levels):
        mid, nf = {}, []
        def m(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                p = v[a] + v[b]
                v.append(p / np.linalg.norm(p))
                mid[key] = len(v) - 1
            return mid[key]
        for a, b, c in f:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        f = nf
    return np.array(v) * radius + np.asarray(center), np.array(f, np.int32)


def test_obj_loader_splits_quads_and_reads_slashed_indices(tmp_path):
    from aether_b200.lua_api import load_obj
    p = tmp_path / "m.obj"
    p.write_text("# cube face\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nv 0 0 1\n"
                 "f 1/1/1 2/2/2 3/3/3 4/4/4\nf 1 2 5\n")
    v, f = load_obj(str(p))
    assert v.shape == (5, 3) and v[2].tolist() == [1, 1, 0]
    assert f.tolist() == [[0, 1, 2], [0, 2, 3], [0, 1, 4]]


@pytest.mark.gpu
@pytest.mark.skipif(not oracle_lib.available("ref"), reason="reference build absent")
@pytest.mark.parametrize("scale", [1.0, 0.5])
def test_gpu_mesh_matches_reference(scale):
    """Add_Mesh: a closed icosphere, scaled, beside a block; the reference
    casts rays in random directions, so cells agree wherever the crossing
    parity does not depend on the ray (here: everywhere)."""
    v, f = icosphere((41.3e-9, 37.7e-9, 33.1e-9), 23.9e-9)
    v = v / scale
    ops = [op(A.OP_BLOCK, 1, 0, 80e-9, 0, 80e-9, 0, 12e-9),
           op(A.OP_MESH, 2, 1e-9, 2e-9, 3e-9, scale, 0)]
    desc = A.structure_desc(0, (0, 0, 0), (0, 0, 0), (80e-9,) * 3, meshes=[(v, f)])
    n = 32
    d = (2.5e-9,) * 3
    ref = oracle_lib.ref_discretize(n, n, n, d, ops, desc)
    gpu = _gpu_discretize(n, n, n, d, ops, desc)
    assert (ref == 2).sum() > 2000
    assert np.array_equal(gpu, ref), np.argwhere(gpu != ref)[:5]
