"""Small seeded scenes used by the parity tests (sizes the oracle finishes in
seconds), covering both drivers, all boundary kinds and every material model."""
from aether_b200 import _abi as A
from aether_b200 import configs as CF


def slab_tm(precision=A.FP64, nsteps=300, **kw):
    return CF.slab_scene(nx=10, ny=8, nz_total=70, pml=8, slab=8, nsteps=nsteps, nl=9, sensor_gap=4,
                         polarization=1, precision=precision, **kw)


def slab_te(precision=A.FP64, nsteps=300):
    return CF.slab_scene(nx=7, ny=9, nz_total=64, pml=6, slab=6, n_slab=2.0, nsteps=nsteps, nl=7,
                         sensor_gap=4, polarization=0, precision=precision)


def gold_sphere(precision=A.FP64, nsteps=300):
    return CF.sphere_scene(nx=12, ny=10, nz_total=90, dx=2.5e-9, pml=8, radius=8e-9, nsteps=nsteps, nl=7,
                           sensor_gap=4, precision=precision)


def debye_lorentz_sphere(precision=A.FP64, nsteps=250):
    mat = A.material_desc(2.2, debye=[(1.3, 2.0e-15)], lorentz=[(0.8, 4.5e15, 3.0e14), (0.3, 6.0e15, 1.0e15)])
    return CF.sphere_scene(nx=11, ny=13, nz_total=84, dx=3e-9, pml=8, radius=9e-9, nsteps=nsteps, nl=5,
                           sensor_gap=4, precision=precision, material=mat)


def custom_box(precision=A.FP64, nsteps=120, n_dielectric=6, seed=7, nl=5):
    return CF.random_spheres_scene(n_total=(40, 36, 44), pml=6, n_dielectric=n_dielectric, n_lorentz=3,
                                   r_range=(10e-9, 30e-9), nsteps=nsteps, nl=nl, precision=precision, seed=seed)


def custom_many_materials(precision=A.FP64, nsteps=80):
    """More than 256 material indices: exercises 16-bit material ids."""
    return CF.random_spheres_scene(n_total=(42, 40, 46), pml=6, n_dielectric=300, n_lorentz=2,
                                   r_range=(4e-9, 12e-9), nsteps=nsteps, nl=4, precision=precision, seed=11)


def thin_column(precision=A.FP64, nsteps=200):
    """Nx = 1: the periodic x wrap reads the cell itself."""
    return CF.slab_scene(nx=1, ny=5, nz_total=60, pml=6, slab=6, nsteps=nsteps, nl=5, sensor_gap=4,
                         precision=precision)


ALL = {
    "slab_tm": slab_tm, "slab_te": slab_te, "gold_sphere": gold_sphere,
    "debye_lorentz_sphere": debye_lorentz_sphere, "custom_box": custom_box,
    "custom_many_materials": custom_many_materials, "thin_column": thin_column,
}
