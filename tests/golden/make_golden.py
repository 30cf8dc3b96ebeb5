"""Generates the golden fixtures from the reference's own FDTD core.

Runs each scene of tests/scenes.py (GOLDEN list) through oracle/_ref/libaeref.so
— the reference sources compiled unmodified by oracle/Makefile — and stores
fields, plane sums, spectra and flux spectra in tests/golden/<name>.npz.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import hashlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import oracle_lib  # noqa: E402
import scenes  # noqa: E402

GOLDEN = ["slab_tm", "slab_te", "gold_sphere", "debye_lorentz_sphere", "custom_box", "thin_column"]
FULL_FIELDS = {"slab_tm", "slab_te", "thin_column"}   # small enough to store whole
SAMPLE_STRIDE = 97


def field_digest(fields):
    """Per-component SHA-256 of the float64 bytes (bit-exactness), L2 norms and
    a strided sample (tolerance checks)."""
    f = np.ascontiguousarray(fields, dtype=np.float64)
    sha = np.array([hashlib.sha256(f[c].tobytes()).hexdigest() for c in range(6)])
    norms = np.sqrt((f.reshape(6, -1) ** 2).sum(axis=1))
    sample = f.reshape(6, -1)[:, ::SAMPLE_STRIDE].copy()
    return sha, norms, sample


def main():
    for name in GOLDEN:
        sc = scenes.ALL[name]()
        r = oracle_lib.run(sc, "ref")
        sha, norms, sample = field_digest(r["fields"])
        out = {"dims": r["dims"], "field_sha256": sha, "field_norms": norms, "field_sample": sample}
        if name in FULL_FIELDS:
            out["fields"] = r["fields"].astype(np.float64)
        if r["plane_sums"] is not None:
            out["plane_sums"] = r["plane_sums"]
            out["spectra"] = r["spectra"]
        for i, f in enumerate(r["flux"]):
            out[f"flux{i}"] = f
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(name, r["dims"][:3], os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
