"""Seeded initial ensembles of spheroids.

The reference draws positions in ``[a, L-a]`` and orientations from a normalised
uniform cube (``initiation_particle_position.f90:301-349``), then sets velocities from
the fluid (``initiation_particle_velocity.f90:76-115``).  The benchmark ensembles use:

* positions uniform in ``[r, L-r]^3`` with ``r`` the largest semi-axis (the
  reference draws in ``[EMAJ, L-EMAJ]``, ``initiation_particle_position.f90:309-316``;
  its wall test runs on the x planes even in periodic mode, so a particle must not
  start across them);
* orientations uniform on S^3 (Shoemake's subgroup algorithm);
* shapes and Stokes numbers per :class:`~gazpart_b200.config.ParticleSpec`;
* per-unit-mass inertia ``IPXX=(b^2+c^2)/5, IPYY=(a^2+c^2)/5, IPZZ=(a^2+b^2)/5``
  (``initiation_particle_position.f90:609-634``);
* translational velocity equal to the interpolated fluid velocity and angular velocity
  equal to half the fluid vorticity expressed in the body frame (set by the caller
  once the field is interpolated, see :func:`body_half_vorticity`).

All draws come from ``numpy.random.default_rng(seed)`` in a fixed order.
"""
from __future__ import annotations

import math
from typing import Dict

import numpy as np

from .config import ParticleSpec, Setup, integral_time, d_equiv

STATE_KEYS = ("x", "y", "z", "u", "v", "w", "qa", "qb", "qc", "qd", "ox", "oy", "oz")
PROP_KEYS = ("emaj", "apr", "rhop", "ipxx", "ipyy", "ipzz")


def draw(spec: ParticleSpec, setup: Setup) -> Dict[str, np.ndarray]:
    """Positions, orientations and properties (velocities zero) of a seeded ensemble."""
    rng = np.random.default_rng(spec.seed)
    n = spec.n
    out: Dict[str, np.ndarray] = {}
    rx, ry, rz = rng.random(n), rng.random(n), rng.random(n)
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    s1, s2 = np.sqrt(1.0 - u1), np.sqrt(u1)
    out["qa"] = s2 * np.cos(2.0 * math.pi * u3)
    out["qb"] = s1 * np.sin(2.0 * math.pi * u2)
    out["qc"] = s1 * np.cos(2.0 * math.pi * u2)
    out["qd"] = s2 * np.sin(2.0 * math.pi * u3)
    if spec.ar is not None:
        ar = np.full(n, float(spec.ar))
    else:
        lo, hi = spec.ar_range
        ar = np.exp(rng.uniform(math.log(lo), math.log(hi), n))
    if spec.b is not None:
        b = np.full(n, float(spec.b))
    else:
        mu, sig = spec.b_lognormal
        b = np.exp(rng.normal(mu, sig, n))
    if spec.st is not None:
        st = np.full(n, float(spec.st))
    elif spec.st_uniform is not None:
        st = rng.uniform(spec.st_uniform[0], spec.st_uniform[1], n)
    else:
        lo, hi = spec.st_loguniform
        st = np.exp(rng.uniform(math.log(lo), math.log(hi), n))
    prolate = ar >= 1.0
    emaj = np.where(prolate, ar * b, b)
    apr = ar.copy()
    deq = (2.0 * emaj) / (apr ** (2.0 / 3.0))
    rhop = st * 18.0 * setup.visc * integral_time() / (deq * deq) * setup.rhof
    if spec.st is not None and spec.ar is not None and spec.b is not None and not spec.density_from_st:
        # monodisperse: exactly the nominal density ratio
        rhop = np.full(n, spec.density_ratio * setup.rhof)
    # positions as the reference draws them, XRAND*(L - 2 EMAJ) + EMAJ
    # (initiation_particle_position.f90:309-316), with the largest semi-axis in place of
    # EMAJ so that no particle starts across the x planes that the wall test watches
    r = np.maximum(emaj, emaj / apr)
    rx_margin = np.maximum(r, spec.x_margin)
    out["x"] = rx * (setup.lx - 2.0 * rx_margin) + rx_margin
    out["y"] = ry * (setup.ly - 2.0 * r) + r
    out["z"] = rz * (setup.lz - 2.0 * r) + r
    out["emaj"] = emaj
    out["apr"] = apr
    out["rhop"] = rhop
    ell_a = emaj
    ell_b = ell_a / apr
    ell_c = ell_b
    out["ipxx"] = (ell_b * ell_b + ell_c * ell_c) / 5.0
    out["ipyy"] = (ell_a * ell_a + ell_c * ell_c) / 5.0
    out["ipzz"] = (ell_a * ell_a + ell_b * ell_b) / 5.0
    for k in ("u", "v", "w", "ox", "oy", "oz"):
        out[k] = np.zeros(n)
    return out


def rotate_to_body(vx, vy, vz, qa, qb, qc, qd):
    """R(conj(q)) v with transform_basis.f90:44-77's expressions and summation order."""
    q0, q1, q2, q3 = qa, -qb, -qc, -qd
    r11 = 1.0 - 2.0 * (q2 * q2 + q3 * q3)
    r12 = 2.0 * (q1 * q2 - q0 * q3)
    r13 = 2.0 * (q1 * q3 + q0 * q2)
    r21 = 2.0 * (q1 * q2 + q0 * q3)
    r22 = 1.0 - 2.0 * (q1 * q1 + q3 * q3)
    r23 = 2.0 * (q2 * q3 - q0 * q1)
    r31 = 2.0 * (q1 * q3 - q0 * q2)
    r32 = 2.0 * (q2 * q3 + q0 * q1)
    r33 = 1.0 - 2.0 * (q1 * q1 + q2 * q2)
    return (r11 * vx + r12 * vy + r13 * vz,
            r21 * vx + r22 * vy + r23 * vz,
            r31 * vx + r32 * vy + r33 * vz)


def body_half_vorticity(st: Dict[str, np.ndarray], vortx, vorty, vortz) -> None:
    """Set omega = 1/2 (fluid vorticity in the body frame), the initial spin."""
    cx, cy, cz = rotate_to_body(vortx, vorty, vortz, st["qa"], st["qb"], st["qc"], st["qd"])
    st["ox"] = 0.5 * cx
    st["oy"] = 0.5 * cy
    st["oz"] = 0.5 * cz
