"""The C-ABI library: loads, exports every entry point include/aefdtd.h
declares, and its struct layouts match the ctypes mirror. No compute calls
unless a GPU is present."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from aether_b200 import _abi as A
from aether_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "aefdtd.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\*?\s*(aefdtd_[a-z_0-9]+)\s*\(", txt, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "aefdtd_create" in names and "aefdtd_step" in names and len(names) >= 20


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert set(declared_functions()) == set(_lib.exported_symbols())


def test_no_cpu_fallback_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = [l.split()[-1] for l in out.splitlines() if " T " in l]
    assert all(n.startswith("aefdtd_") for n in exported if not n.startswith("_")), exported


def test_struct_layouts_match_header():
    src = """
#include <stdio.h>
#include <stddef.h>
#include "aefdtd.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(aefdtd_grid_desc), sizeof(aefdtd_material_desc),
         sizeof(aefdtd_normal_desc), sizeof(aefdtd_sensor_desc), sizeof(aefdtd_source_desc),
         sizeof(aefdtd_dims), sizeof(aefdtd_structure_op));
  printf("%zu %zu %zu\\n", offsetof(aefdtd_grid_desc, pml_kappa), offsetof(aefdtd_grid_desc, dft_block),
         offsetof(aefdtd_material_desc, critpoint));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in lines[0].split()]
    offs = [int(x) for x in lines[1].split()]
    assert sizes == [C.sizeof(A.GridDesc), C.sizeof(A.MaterialDesc), C.sizeof(A.NormalDesc),
                     C.sizeof(A.SensorDesc), C.sizeof(A.SourceDesc), C.sizeof(A.Dims), C.sizeof(A.StructureOp)]
    assert offs == [A.GridDesc.pml_kappa.offset, A.GridDesc.dft_block.offset, A.MaterialDesc.critpoint.offset]


def test_status_strings():
    lib = _lib.load()
    for st in range(7):
        assert lib.aefdtd_status_string(st)


def test_bad_descriptor_rejected_before_device_use():
    lib = _lib.load()
    h = C.c_void_p()
    g = A.grid_desc(8, 8, 8, 5e-9)
    g.abi_version = 999
    st = lib.aefdtd_create(C.byref(g), C.byref(h))
    assert st in (1, 6)  # BAD_ARG, or NO_DEVICE where no GPU is visible
    assert not h


def test_create_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    lib = _lib.load()
    h = C.c_void_p()
    g = A.grid_desc(8, 8, 8, 5e-9)
    assert lib.aefdtd_create(C.byref(g), C.byref(h)) == 6


SHIM_SRC = r"""
#include <cstdio>
#include <vector>
#include "aefdtd.hpp"
int main() {
    try {
        // 24 x 20 x 40 structure at 5 nm, CPML 8 on z, vacuum with an n = 1.5 block
        aefdtd::FDTD f(24, 20, 40, 400, 5e-9, 5e-9, 5e-9, 0.0, "NORMAL", 0, 0, 0, 0, 8, 8, 0, 0, 0, 0, 5, 5);
        f.set_pml_zm(1.0, 1.0, 0.05);
        f.set_pml_zp(1.0, 1.0, 0.05);
        f.set_time_mod(0.5 / 0.99);
        f.bootstrap();
        std::vector<uint32_t> map(24 * 20 * 40, 0);
        for (int k = 15; k < 25; k++)
            for (int j = 0; j < 20; j++)
                for (int i = 0; i < 24; i++) map[i + 24 * (j + 20 * k)] = 1;
        f.set_matsgrid(map);
        aefdtd_material_desc vac{}, diel{};
        vac.eps_inf = 1.0;
        diel.eps_inf = 2.25;
        f.set_material(0, vac);
        f.set_material(1, diel);
        aefdtd_normal_desc nd{};
        nd.polarization = 1; nd.nl = 11; nd.lambda_min = 400e-9; nd.lambda_max = 1000e-9;
        f.setup_normal(nd);
        f.update(60);
        std::vector<double> ex = f.get_field(0);
        double s = 0;
        for (double v : ex) s += v * v;
        std::printf("ok %d %.17g\n", f.tstep(), s);
    } catch (const aefdtd::Error &e) {
        std::printf("error %d %s\n", (int)e.status, e.what());
    }
    return 0;
}
"""


def build_shim_program(d):
    src = os.path.join(d, "shim.cpp")
    open(src, "w").write(SHIM_SRC)
    exe = os.path.join(d, "shim")
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.dirname(HEADER), src, "-o", exe, "-L", libdir,
                    "-laefdtd", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def shim_scene():
    """The structure, materials and excitation the shim program builds."""
    import numpy as np
    from aether_b200.scene import Scene
    g = A.grid_desc(24, 20, 40, 5e-9, mode=A.MODE_NORMAL, precision=A.FP64, nt=400, pml=(0, 0, 0, 0, 8, 8),
                    pad=(0, 0, 0, 0, 5, 5), time_mod=0.5 / 0.99, alpha=(0, 0, 0, 0, 0.05, 0.05))
    m = np.zeros((40, 20, 24), np.uint32)
    m[15:25] = 1
    return Scene(g, m, [A.material_desc(1.0), A.material_desc(2.25)], 60,
                 normal=A.NormalDesc(1, 11, 400e-9, 1000e-9), sensors=[], name="shim")


def test_cpp_shim_compiles_and_reports_no_device_without_gpu():
    """The FDTD-named C++ shim builds against the C ABI; without a GPU its
    first use throws AEFDTD_NO_DEVICE (there is no CPU path)."""
    import torch
    with tempfile.TemporaryDirectory() as d:
        exe = build_shim_program(d)
        if torch.cuda.is_available():
            pytest.skip("GPU present: covered by the gpu test")
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
        assert out.startswith("error 6"), out


def test_batch_and_server_struct_layouts_match_header():
    src = """
#include <stdio.h>
#include <stddef.h>
#include "aefdtd.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(aefdtd_batch_opts), sizeof(aefdtd_batch_info),
         sizeof(aefdtd_server_opts), sizeof(aefdtd_job_desc), sizeof(aefdtd_job_info), sizeof(aefdtd_server_stats));
  printf("%zu %zu %zu %zu\\n", offsetof(aefdtd_batch_info, class_kchunk), offsetof(aefdtd_server_opts, batch),
         offsetof(aefdtd_job_desc, steps), offsetof(aefdtd_server_stats, gcells_per_s));
  printf("%zu %zu\\n", sizeof(aefdtd_box_sensor_desc), offsetof(aefdtd_box_sensor_desc, lambda_min));
  printf("%zu %zu %zu\\n", sizeof(aefdtd_fieldmap_desc), offsetof(aefdtd_fieldmap_desc, magnetic),
         offsetof(aefdtd_fieldmap_desc, lambda));
  printf("%zu %zu\\n", sizeof(aefdtd_oblique_desc), offsetof(aefdtd_oblique_desc, kx_in));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in lines[0].split()]
    offs = [int(x) for x in lines[1].split()]
    assert sizes == [C.sizeof(A.BatchOpts), C.sizeof(A.BatchInfo), C.sizeof(A.ServerOpts), C.sizeof(A.JobDesc),
                     C.sizeof(A.JobInfo), C.sizeof(A.ServerStats)]
    assert offs == [A.BatchInfo.class_kchunk.offset, A.ServerOpts.batch.offset, A.JobDesc.steps.offset,
                    A.ServerStats.gcells_per_s.offset]
    assert [int(x) for x in lines[2].split()] == [C.sizeof(A.BoxSensorDesc), A.BoxSensorDesc.lambda_min.offset]
    assert [int(x) for x in lines[3].split()] == [C.sizeof(A.FieldMapDesc), A.FieldMapDesc.magnetic.offset,
                                                  A.FieldMapDesc.lambda_.offset]
    assert [int(x) for x in lines[4].split()] == [C.sizeof(A.ObliqueDesc), A.ObliqueDesc.kx_in.offset]
