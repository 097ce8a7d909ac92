"""What the oracle's choices on the collision path change, measured on the CPU.

1. Trigonometry of the contact solve.  The reference calls libm's sin, cos, asin and acos
   in ellipsoid_contact_detection (ellipsoid_contact_detection.f90:77-87,193-334).  The
   oracle and the device share their own (Cody-Waite reduction by fdlibm's three-part
   pi/2, Taylor polynomials) so that their Levenberg-Marquardt iterates agree bit for
   bit.  The same restatement built with libm's functions (libgazpart_oracle_libm.so)
   shows what that choice changes: no contact flag on 4,000 pairs like those of the
   512^3 workload, a few evaluation counts, and no accepted pair over 20 steps of the dense and polydisperse
   cases.
2. The prefilters.  The reference solves every candidate pair (Q12); the oracle and the
   device first drop pairs whose bodies are provably apart.  On the dense, polydisperse
   and bimodal cases, before and after 10 steps, the accepted pairs and the states are
   the same with and without them.
3. How an ulp of input moves a collision.  A contact solve stops at xtol = sqrt(eps) of
   its angles; changing its inputs by one ulp can change where it stops, so a collided
   particle's velocity moves by much more than an ulp while the pair set stays put.  This
   is why a device step, whose advance differs from the oracle's by a few ulps (libm pow,
   atan, sin, cos), leaves collided particles further from the oracle than free ones."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle as po
from _cases import case, copy_state, rel_err

STATE = po.STATE_KEYS


def _c3_pairs(n, seed):
    """Pairs at the 512^3/16.8M workload's shapes: minor semi-axis log-normal around 1e-3,
    aspect ratio log-uniform in [0.2, 5], centres from deep overlap to just touching."""
    rng = np.random.default_rng(seed)
    b = np.exp(rng.normal(np.log(1e-3), 0.3, (n, 2)))
    ar = np.exp(rng.uniform(np.log(0.2), np.log(5.0), (n, 2)))
    emaj = np.where(ar >= 1, ar * b, b)
    q = rng.normal(size=(n, 8))
    q[:, :4] /= np.linalg.norm(q[:, :4], axis=1, keepdims=True)
    q[:, 4:] /= np.linalg.norm(q[:, 4:], axis=1, keepdims=True)
    b1 = rng.uniform(1.0, 2.0, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    reach = np.maximum(emaj[:, 0], emaj[:, 0] / ar[:, 0]) + np.maximum(emaj[:, 1], emaj[:, 1] / ar[:, 1])
    b2 = b1 + d * (reach * rng.uniform(0.2, 1.0, n))[:, None]
    return emaj, ar, b1, b2, q


def test_shared_trigonometry_against_libm_contact_decisions():
    n = 4000
    emaj, ar, b1, b2, q = _c3_pairs(n, 3)
    flags = np.zeros((2, n), dtype=int)
    nfev = np.zeros((2, n), dtype=int)
    ept = np.zeros((2, n, 3))
    for i in range(n):
        for v, var in enumerate(("shared", "libm")):
            r = po.contact_detection(emaj[i, 0], ar[i, 0], emaj[i, 1], ar[i, 1], b1[i], q[i, :4], b2[i], q[i, 4:],
                                     variant=var)
            flags[v, i], nfev[v, i], ept[v, i] = r["flag"], r["nfev"], r["ept1"]
    assert 0.2 * n < flags[0].sum() < 0.8 * n
    assert np.array_equal(flags[0], flags[1])                 # no contact decision changes
    changed = int((nfev[0] != nfev[1]).sum())
    assert changed <= n // 200                                # iteration paths almost never change
    finite = ~np.isnan(ept[0, :, 0])
    exact = np.all(ept[0] == ept[1], axis=1) & finite
    assert exact.sum() > 0.5 * finite.sum()                   # most contact points are bit-identical
    print(f"\n{n} pairs: 0 flags differ, {changed} evaluation counts differ, "
          f"{int(exact.sum())} of {int(finite.sum())} contact points bit-identical")


@pytest.mark.parametrize("name", ["dense", "poly"])
def test_shared_trigonometry_against_libm_pair_sets(name):
    setup, fn, refs, st = case(name)
    runs = {}
    for var in ("shared", "libm"):
        ens = po.Ensemble(setup, copy_state(st), variant=var)
        pairs = []
        for _ in range(20):
            assert ens.advance(refs, nthreads=8) == 0
            r = ens.collide(prefilter=True, nthreads=8)
            assert r["rc"] == 0
            pairs.append((r["home"], r["near"], r["n_contacts"]))
        runs[var] = (pairs, {k: ens.a[k].copy() for k in STATE})
    for (h0, n0, c0), (h1, n1, c1) in zip(runs["shared"][0], runs["libm"][0]):
        assert np.array_equal(h0, h1) and np.array_equal(n0, n1) and c0 == c1
    assert rel_err(runs["shared"][1], runs["libm"][1], STATE) < 1e-9


@pytest.mark.parametrize("name", ["dense", "poly", "bimodal_small"])
def test_prefilter_changes_no_pair(name):
    """collision_interaction.f90:190-419 solves every candidate pair; with the exact
    prefilters (non-overlapping bounding spheres, separation along the centre line or
    along a support-function ascent direction) the result is the same."""
    setup, fn, refs, st = case(name)
    ens = po.Ensemble(setup, copy_state(st))
    collisions = 0
    for check_step in (0, 10):
        while check_step > 0:
            assert ens.advance(refs, nthreads=8) == 0
            assert ens.collide(prefilter=True, nthreads=8)["rc"] == 0
            check_step -= 1
        a = po.Ensemble(setup, {**{k: ens.a[k] for k in STATE + po.PROP_KEYS}})
        b = po.Ensemble(setup, {**{k: ens.a[k] for k in STATE + po.PROP_KEYS}})
        ra = a.collide(prefilter=True, nthreads=8)
        rb = b.collide(prefilter=False, nthreads=8)
        assert ra["rc"] == 0 and rb["rc"] == 0
        assert np.array_equal(ra["home"], rb["home"]) and np.array_equal(ra["near"], rb["near"])
        assert ra["n_contacts"] == rb["n_contacts"]
        for k in STATE:
            assert np.array_equal(a.a[k], b.a[k]), k
        collisions += rb["n_coll"]
    assert collisions > 0


def test_one_ulp_of_input_moves_collided_particles_only():
    """The dense case, advanced once, then collided from that state and from the same
    state with every position and quaternion component moved by one ulp.  Pair sets are
    the same; particles in no collision keep the one-ulp difference; collided particles
    differ by more than an ulp (the contact solve's stopping point moves), but stay far
    inside 1e-9."""
    setup, fn, refs, st = case("dense")
    ens = po.Ensemble(setup, copy_state(st))
    assert ens.advance(refs, nthreads=8) == 0
    s1 = {k: ens.a[k].copy() for k in STATE + po.PROP_KEYS}
    pert = dict(s1)
    for k in ("x", "y", "z", "qa", "qb", "qc", "qd"):
        pert[k] = np.nextafter(s1[k], np.inf)
    a, b = po.Ensemble(setup, s1), po.Ensemble(setup, pert)
    ra, rb = a.collide(prefilter=True, nthreads=8), b.collide(prefilter=True, nthreads=8)
    assert np.array_equal(ra["home"], rb["home"]) and np.array_equal(ra["near"], rb["near"])
    hit = np.zeros(a.n, dtype=bool)
    hit[ra["home"]] = True
    hit[ra["near"]] = True
    free = rel_err({k: a.a[k][~hit] for k in STATE}, {k: b.a[k][~hit] for k in STATE}, STATE)
    coll = rel_err({k: a.a[k][hit] for k in STATE}, {k: b.a[k][hit] for k in STATE}, STATE)
    assert free < 1e-15
    assert 1e-15 < coll < 1e-9, coll
    print(f"\none ulp in: free particles {free:.1e}, collided particles {coll:.1e}")
