"""The oblique driver's wavevector sweep ("fdtd_oblique_ARS",
FDTD_oblique_biphase, oblique_biphase.cpp:645-680): one simulation per in-plane
wavevector kp, at kx = kp cos(phi), ky = kp sin(phi).

`kp_list` restates FDTD_oblique_biphase_get_kp (oblique_biphase.cpp:503-597)
for the Lua setters kp_auto, kp_full, kp_fixed_angle, kp_fixed_lambda and
kp_target (lua_fdtd.cpp:554-634); `sweep` runs the list on the GPU and returns
the rows the driver writes to its obl_<m> files."""
from __future__ import annotations

import math
from typing import List

from . import _abi as A
from . import fdtd


def kp_list(kind: str, *, lambda_min=None, lambda_max=None, amin_deg=0.0, amax_deg=0.0, nkp=1, kp_ic=0.0,
            kp_fc=1.0, lmin=500e-9, lmax=500e-9) -> List[float]:
    """In-plane wavevectors (rad/m in vacuum) of one sweep.

    kind "auto" (kp_auto(amin, amax)): geometric series between the driver's
    lambda_max and lambda_min; "full" (kp_full(Nkp, kp_ic, kp_fc)); "fixed_angle"
    (kp_fixed_angle(Nkp, lmin, lmax, angle)); "fixed_lambda"
    (kp_fixed_lambda(Nkp, lambda, amin, amax)); "target" (kp_target(lambda,
    angle)). Angles in degrees as in the Lua setters, which store
    degrees * Pi / 180."""
    Pi = math.pi
    amin = amin_deg * Pi / 180.0
    amax = amax_deg * Pi / 180.0
    if kind == "auto":
        nk = 1
        tfsin = math.sin(amin) / math.sin(amax)
        tmpl = lambda_max * tfsin
        while tmpl > lambda_min:
            tmpl = tmpl * tfsin
            nk += 1
        out = []
        for m in range(nk):
            kp = 2.0 * Pi / lambda_max * math.sin(amax)
            for _ in range(m):
                kp *= math.sin(amax) / math.sin(amin)
            out.append(kp)
        return out
    if kind == "full":
        kp_fc = min(max(kp_fc, 0.0), 0.95)
        kp_ic = min(max(kp_ic, 0.0), kp_fc)
        out = []
        for m in range(nkp):
            m_ct = m / (nkp - 1.0) if nkp > 1 else 1.0
            m_c = 0.99 * Pi / 2.0 * (kp_ic + (kp_fc - kp_ic) * m_ct)
            m_lambda = lambda_min + math.cos(m_c) * (lambda_max - lambda_min)
            m_ang = Pi / 2.0 * math.sin(m_c)
            out.append(2.0 * Pi / m_lambda * math.sin(m_ang))
        return out
    if kind == "fixed_angle":
        return [2.0 * Pi / (lmax + (lmin - lmax) * m / (nkp - 1.0)) * math.sin(amin) for m in range(nkp)]
    if kind == "fixed_lambda":
        return [2.0 * Pi / lmin * math.sin(amin + (amax - amin) * i / (nkp - 1.0)) for i in range(nkp)]
    if kind == "target":
        return [2.0 * Pi / lmin * math.sin(amin)]
    raise ValueError(f"unknown kp sweep kind {kind!r}")


def sweep(scene, kps, phi_deg=0.0, nsteps=None, batch=False, hbm_fraction=0.8, max_chunk=0):
    """Runs `scene` (mode OBLIQUE) once per kp at kx = kp cos(phi), ky = kp
    sin(phi) (incident_plane(phi), stored as Degree(phi)); returns one
    (nl', 10) array per kp: lambda, angle, |r_TE|, arg, |r_TM|, arg, |t_TE|,
    arg, |t_TM|, arg. batch=True advances the wavevectors together in batches
    (each as a subset of its own, two at a time on the GPU) with the same
    results. A batch holds as many wavevectors as fit: members are built one
    by one while the device's used memory stays within hbm_fraction of its
    total with room for one more member of the first member's footprint
    (max_chunk > 0 caps the count too); the rest run in the next batch. A
    first member that does not fit fails like a single run would."""
    phi = phi_deg * (math.pi / 180.0)
    base = scene.oblique
    steps = scene.nsteps if nsteps is None else nsteps

    def member(kp):
        scene.oblique = A.ObliqueDesc(base.polarization, base.nl, base.lambda_min, base.lambda_max,
                                      kp * math.cos(phi), kp * math.sin(phi))
        try:
            return fdtd.build_simulation(scene)
        finally:
            scene.oblique = base

    if batch:
        out = []
        while len(out) < len(kps):
            sims = []
            try:
                while len(out) + len(sims) < len(kps) and (max_chunk <= 0 or len(sims) < max_chunk):
                    if sims:
                        free, total = fdtd.device_memory(scene.grid.device)
                        per = sims[0].dims().device_bytes
                        if (total - free) + per > hbm_fraction * total:
                            break
                    sims.append(member(kps[len(out) + len(sims)]))
                with fdtd.Batch() as b:
                    for s in sims:
                        b.add(s, steps)
                    b.run(10 ** 9)
                    out.extend(s.oblique_spectra() for s in sims)
            finally:
                for s in sims:
                    s.close()
        return out
    out = []
    for kp in kps:
        od = A.ObliqueDesc(base.polarization, base.nl, base.lambda_min, base.lambda_max,
                           kp * math.cos(phi), kp * math.sin(phi))
        scene.oblique = od
        try:
            with fdtd.build_simulation(scene) as s:
                s.step(steps)
                out.append(s.oblique_spectra())
        finally:
            scene.oblique = base
    return out
