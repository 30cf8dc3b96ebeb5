"""aether_b200 — B200-native 3D FDTD time-stepping core with Aether's FDTD
mode, structure, material and sensor surface.

The compute path is the CUDA library aether_b200/libaefdtd.so behind the C ABI
of include/aefdtd.h; this package is its Python binding and scripting surface."""
