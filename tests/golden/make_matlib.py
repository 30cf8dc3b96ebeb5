"""Generates tests/golden/mat_lib.json from the reference's material library.

Reads every mat_lib/*.lua file of the reference tree (AEFDTD_REFERENCE, or the
default location below) with aether_b200.matlib and records, per file,
whether the FDTD can use it ("loaded") or not ("refused", with the reason),
its eps_inf, its terms in call order and its name. The GPU tests use the
recorded terms, so they need no reference tree at run time.

    python tests/golden/make_matlib.py
"""
import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from aether_b200 import matlib  # noqa: E402

REFERENCE = os.environ.get("AEFDTD_REFERENCE", "/root/reference")


def record(path):
    m = matlib.load_file(path)
    why = m.refusal()
    return {"status": "refused" if why else "loaded", "reason": why, "eps_inf": m.eps_inf,
            "terms": {k: [list(t) for t in v] for k, v in m.terms.items()}, "name": m.name}


def main():
    files = sorted(glob.glob(os.path.join(REFERENCE, "mat_lib", "*.lua")))
    if not files:
        sys.exit(f"no material files under {REFERENCE}/mat_lib")
    out = {os.path.basename(f): record(f) for f in files}
    with open(os.path.join(HERE, "mat_lib.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"{len(out)} files: {sum(v['status'] == 'loaded' for v in out.values())} loaded, "
          f"{sum(v['status'] == 'refused' for v in out.values())} refused")


if __name__ == "__main__":
    main()
