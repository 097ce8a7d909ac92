"""Generate tests/golden/lm_contact.json: contact problems solved by scipy's MINPACK.

The reference solves the ellipsoid contact problem with a vendored copy of MINPACK's
lmder (minpack_reduc.f90, called through lmder1 from ellipsoid_contact_detection.f90:92
with ftol = xtol = sqrt(eps), gtol = 0, maxfev = 300).  scipy.optimize.leastsq wraps
the same MINPACK routine.  This script restates the residual and Jacobian of
ellipsoid_contact_detection.f90:193-334 in numpy (independently of the oracle), runs
leastsq from the reference's initial guess, and records inputs and outputs.

Run from the repository root:  python tests/golden/make_lm_golden.py
"""
from __future__ import annotations

import json
import os

import numpy as np
from scipy.optimize import leastsq

HERE = os.path.dirname(os.path.abspath(__file__))


def rot(q):
    q0, q1, q2, q3 = q
    return np.array([[1 - 2 * (q2 * q2 + q3 * q3), 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
                     [2 * (q1 * q2 + q0 * q3), 1 - 2 * (q1 * q1 + q3 * q3), 2 * (q2 * q3 - q0 * q1)],
                     [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1 - 2 * (q1 * q1 + q2 * q2)]])


def ell(a, apr, q):
    b = a / apr
    R = rot(q)
    return R @ np.diag([a * a, b * b, b * b]) @ R.T


def geometry(x, E1, E2, b1, b2):
    c1 = np.array([np.cos(x[0]) * np.cos(x[1]), np.sin(x[0]) * np.cos(x[1]), np.sin(x[1])])
    c2 = -c1
    l1 = np.sqrt(0.25 * c1 @ E1 @ c1)
    l2 = np.sqrt(0.25 * c2 @ E2 @ c2)
    p1 = E1 @ c1 / (2 * l1) + b1
    p2 = E2 @ c2 / (2 * l2) + b2
    return c1, l1, l2, p1, p2


def residual(x, E1, E2, b1, b2):
    _, _, _, p1, p2 = geometry(x, E1, E2, b1, b2)
    d = p1 - p2
    return d * d


def jacobian(x, E1, E2, b1, b2):
    c1, l1, l2, p1, p2 = geometry(x, E1, E2, b1, b2)
    d = p1 - p2
    G = np.array([[-np.sin(x[0]) * np.cos(x[1]), -np.cos(x[0]) * np.sin(x[1])],
                  [np.cos(x[0]) * np.cos(x[1]), -np.sin(x[0]) * np.sin(x[1])],
                  [0.0, np.cos(x[1])]])
    def coeff(E, c, l):
        return E / (2 * l) - (E @ np.outer(c, c) @ E) / (8 * l ** 3)
    gd = coeff(E1, c1, l1) @ G - coeff(E2, -c1, l2) @ (-G)
    return 2.0 * d[:, None] * gd


def main(n: int = 64, seed: int = 2024):
    rng = np.random.default_rng(seed)
    tol = float(np.sqrt(np.finfo(float).eps))
    cases = []
    while len(cases) < n:
        a1, a2 = rng.uniform(0.004, 0.02, 2)
        p1, p2 = rng.uniform(0.3, 4.0, 2)
        q1 = rng.normal(size=4); q1 /= np.linalg.norm(q1)
        q2 = rng.normal(size=4); q2 /= np.linalg.norm(q2)
        b1 = rng.uniform(0, 1, 3)
        d = rng.normal(size=3); d /= np.linalg.norm(d)
        r = max(a1, a1 / p1) + max(a2, a2 / p2)
        b2 = b1 + d * r * rng.uniform(0.2, 1.1)
        cn = (b1 - b2) / np.linalg.norm(b1 - b2)
        x0 = np.array([np.arccos(cn[0] / np.cos(np.arcsin(cn[2]))), np.arcsin(cn[2])])
        if np.isnan(x0).any():
            continue
        E1, E2 = ell(a1, p1, q1), ell(a2, p2, q2)
        xs, _, info, _, ier = leastsq(residual, x0.copy(), args=(E1, E2, b1, b2), Dfun=jacobian, full_output=True,
                                      ftol=tol, xtol=tol, gtol=0.0, maxfev=300, factor=100)
        c1, _, _, pt1, pt2 = geometry(xs, E1, E2, b1, b2)
        cases.append({"emaj1": a1, "apr1": p1, "emaj2": a2, "apr2": p2, "b1": b1.tolist(), "b2": b2.tolist(),
                      "q1": q1.tolist(), "q2": q2.tolist(), "x0": x0.tolist(), "x": xs.tolist(),
                      "info": int(4 if ier == 8 else ier), "nfev": int(info["nfev"]),
                      "contact": float((pt1 - pt2) @ c1)})
    with open(os.path.join(HERE, "lm_contact.json"), "w") as fh:
        json.dump({"generator": "scipy.optimize.leastsq (MINPACK lmder), numpy residual/Jacobian",
                   "tol": tol, "cases": cases}, fh, indent=1)


if __name__ == "__main__":
    main()
