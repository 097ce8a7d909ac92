"""Parity of the CUDA path (through the C ABI) with the oracle."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle as po
from gazpart_b200 import api
from _cases import REL_TOL, case, copy_state, rel_err

pytestmark = pytest.mark.gpu


def _ctx(setup, fn, st, precision="fp64", store_fluid=False):
    ctx = api.Context(setup, precision, store_fluid=store_fluid)
    ctx.set_fields(fn)
    ctx.upload(st)
    return ctx


def test_interp_lag3_bit_exact():
    setup, fn, refs, st = case("c1")
    rng = np.random.default_rng(3)
    n = 50000
    x, y, z = (rng.random(n) * setup.lx for _ in range(3))
    with api.Context(setup, "fp64") as ctx:
        ctx.set_fields(fn)
        for c in range(6):
            got = ctx.interp_lag3(c, x, y, z)
            ref = po.interp_lag3(setup, refs[c], x, y, z)
            assert np.array_equal(got, ref), (c, np.max(np.abs(got - ref)))
        ctx.raise_status()


def test_interp_reference_layout_source():
    setup, fn, refs, st = case("c1")
    rng = np.random.default_rng(4)
    x, y, z = (rng.random(2000) * setup.lx for _ in range(3))
    with api.Context(setup, "fp64") as ctx:
        for c in range(6):
            ctx.set_field(c, refs[c], layout="reference")
        for c in range(6):
            assert np.array_equal(ctx.interp_lag3(c, x, y, z), po.interp_lag3(setup, refs[c], x, y, z))


def test_one_step_advance():
    setup, fn, refs, st = case("c1")
    ens = po.Ensemble(setup, copy_state(st))
    assert ens.advance(refs) == 0
    with _ctx(setup, fn, st, store_fluid=True) as ctx:
        ctx.adv_particle_ellp(1)
        ctx.raise_status()
        got = ctx.download(fluid=True)
    assert rel_err(got, ens.a, api.STATE_KEYS) < 1e-14
    for k in api.FLUID_KEYS:
        assert np.array_equal(got[k], ens.a[k]), k


@pytest.mark.parametrize("name", ["dense", "poly", "c1", "bimodal"])
def test_collision_pairs_bit_exact(name):
    """Same pre-collision state -> identical accepted pairs in identical order."""
    setup, fn, refs, st = case(name)
    ens = po.Ensemble(setup, copy_state(st))
    res = ens.collide(prefilter=True, nthreads=1)          # the reference's serial walk
    assert res["rc"] == 0
    par = po.Ensemble(setup, copy_state(st)).collide(prefilter=True, nthreads=8)  # evaluates every pair
    assert np.array_equal(par["home"], res["home"]) and np.array_equal(par["near"], res["near"])
    with _ctx(setup, fn, st) as ctx:
        cnt = ctx.collision(1, 0.0)
        ctx.raise_status()
        home, near = ctx.collision_pairs()
        got = ctx.download()
    assert cnt["n_contact"] == par["n_contacts"]
    assert home.size == res["n_coll"]
    if name == "bimodal":   # the large particles (the last 12) take part in collisions
        assert np.any(home >= ens.n - 12) or np.any(near >= ens.n - 12)
    assert np.array_equal(home, res["home"]) and np.array_equal(near, res["near"])
    assert rel_err(got, ens.a, api.STATE_KEYS) < REL_TOL


@pytest.mark.parametrize("name", ["c1", "poly"])
def test_hundred_steps(name):
    """100-step trajectories run freely on both sides: <= 1e-12 relative for every
    particle that has not collided, 1e-9 for all.

    The device's advance differs from the oracle's by a few ulps: the force, torque and
    quaternion routines call pow, atan, sin and cos, and the device's math library and
    the host's differ there in the last bit.  The contact solve itself is identical on
    both sides (shared trigonometry, IEEE operations; test_step_parity checks it bit for
    bit from the same state), but where a Levenberg-Marquardt solve stops (xtol =
    sqrt(eps)) moves with its inputs: one ulp of input moves a collided particle by about
    1e-12 (test_oracle_trig), and along a free trajectory those differences compound
    from collision to collision.  Pair sets from the same state are compared exactly in
    test_collision_pairs_bit_exact and, every step, in test_step_parity."""
    setup, fn, refs, st = case(name)
    ens = po.Ensemble(setup, copy_state(st))
    worst_free = worst_all = 0.0
    collided = np.zeros(ens.n, dtype=bool)
    with _ctx(setup, fn, st) as ctx:
        for step in range(100):
            assert ens.advance(refs, nthreads=8) == 0
            res = ens.collide(prefilter=True, nthreads=8)
            assert res["rc"] == 0
            collided[res["home"]] = True
            collided[res["near"]] = True
            ctx.step(1)
            if step % 10 == 9 or step == 0:
                got = ctx.download()
                free = {k: v[~collided] for k, v in got.items()}
                ref_free = {k: ens.a[k][~collided] for k in api.STATE_KEYS}
                worst_free = max(worst_free, rel_err(free, ref_free, api.STATE_KEYS))
                worst_all = max(worst_all, rel_err(got, ens.a, api.STATE_KEYS))
        ctx.raise_status()
    assert worst_free < REL_TOL, worst_free
    assert worst_all < 1e-9, worst_all


def test_graph_step_matches_api_calls():
    setup, fn, refs, st = case("poly")
    with _ctx(setup, fn, st) as a, _ctx(setup, fn, st) as b:
        for i in range(5):
            a.adv_particle_ellp(i)
            a.collision(i, 0.0)
        b.step(5)
        ga, gb = a.download(), b.download()
    for k in api.STATE_KEYS:
        assert np.array_equal(ga[k], gb[k]), k


@pytest.mark.parametrize("name", ["poly", "dense"])
def test_mixed_precision_error_budget(name):
    """The mixed form (FP32 field and stencil weights, FP32 drag/lift/torque
    coefficients, FP64 integration and contact solve) against the FP64 oracle.

    Free run, 50 steps on each side: the velocity of every particle that collided in
    neither run within 1e-5 relative (the maximum, not a quantile).  Every step the same
    state is also stepped once by the mixed device and the oracle: their accepted pairs
    are compared; a pair decided by the last bits of the positions may flip, and the flips
    are counted and held to 1% of the accepted pairs."""
    setup, fn, refs, st = case(name)
    ens = po.Ensemble(setup, copy_state(st))
    collided = np.zeros(ens.n, dtype=bool)
    mism = accepted = 0
    with _ctx(setup, fn, st, precision="mixed") as free, _ctx(setup, fn, st, precision="mixed") as seeded:
        for step in range(50):
            s0 = {k: ens.a[k].copy() for k in api.STATE_KEYS}
            seeded.put_state(s0)
            seeded.step(1)
            sh, sn = seeded.collision_pairs()
            free.step(1)
            fh, fnr = free.collision_pairs()
            collided[fh] = True
            collided[fnr] = True
            assert ens.advance(refs, nthreads=8) == 0
            r = ens.collide(prefilter=True, nthreads=8)
            assert r["rc"] == 0
            collided[r["home"]] = True
            collided[r["near"]] = True
            a = set(zip(sh.tolist(), sn.tolist()))
            b = set(zip(r["home"].tolist(), r["near"].tolist()))
            mism += len(a ^ b)
            accepted += len(b)
        free.raise_status()
        seeded.raise_status()
        got = free.download()
    du = np.sqrt(sum((got[k] - ens.a[k]) ** 2 for k in ("u", "v", "w")))
    nu = np.sqrt(sum(ens.a[k] ** 2 for k in ("u", "v", "w")))
    err = du / (nu + 1e-30)
    free_err = float(np.max(err[~collided]))
    print(f"\n{name}: mixed vs FP64 oracle after 50 steps: max {free_err:.2e} over {int((~collided).sum())} "
          f"never-collided particles (all: median {np.median(err):.1e}, max {err.max():.1e}); "
          f"pairs from the same state: {mism} flips in {accepted} accepted")
    assert free_err < 1e-5
    assert accepted > 0
    assert mism <= max(1, accepted // 100)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["dense", "bimodal"])
def test_speculative_integrate_changes_nothing(name, precision):
    """Step s+1's integrate run on the side stream beside step s's contact solves for
    the particles in none of step s's candidate pairs, and after the response for the
    pair members, gives the state of the plain order bit for bit: one six-step graph,
    five of its steps speculative, against the same graph without any overlap and with
    the gather alone overlapped."""
    setup, fn, refs, st = case(name)
    grids = {"gather": 296, "integrate": 592, "bin": 592, "search": 592}
    out = {}
    for mode in ("plain", "gather", "spec"):
        with _ctx(setup, fn, st, precision) as ctx:
            ctx.set_launch({**grids, "overlap_gather": mode != "plain", "speculative_integrate": mode == "spec"})
            ctx.step(6)
            ctx.raise_status()
            out[mode] = (ctx.download(), ctx.collision_counters())
    assert out["plain"][1]["accepted"] > 0
    for mode in ("gather", "spec"):
        assert out[mode][1] == out["plain"][1], mode
        for k in api.STATE_KEYS:
            assert np.array_equal(out[mode][0][k], out["plain"][0][k]), (mode, k)


@pytest.mark.parametrize("name", ["dense", "bimodal"])
def test_contact_tail_hand_over_changes_nothing(name):
    """Solves handed from one pass of the contact kernel to the next (gp_set_contact_tail)
    run the same iterates: with every solve handed on after 1, 3, 9, ... evaluations
    (seven passes), after 4, 12, 36, 108, after 64 and 192, and with one pass, the
    colliding pairs, the counters and the states after a step are identical."""
    setup, fn, refs, st = case(name)
    res = po.Ensemble(setup, copy_state(st)).collide(prefilter=True, nthreads=8)
    out = {}
    for budget in (0, 1, 4, 64):
        with _ctx(setup, fn, st) as ctx:
            ctx.set_contact_tail(budget)
            ctx.collision(1, 0.0)
            ctx.raise_status()
            out[budget] = (ctx.collision_pairs(), ctx.download(), ctx.collision_counters())
    for budget in (0, 1, 4, 64):
        (home, near), got, cnt = out[budget]
        assert np.array_equal(home, res["home"]) and np.array_equal(near, res["near"]), budget
        for k in api.STATE_KEYS:
            assert np.array_equal(got[k], out[0][1][k]), (budget, k)
        assert cnt == out[0][2], budget


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["dense", "bimodal"])
def test_contact_order_changes_nothing(name, precision):
    """The contact queue's order (solves handed out in decreasing predicted length, from
    what each particle's solves took in the last collision phase) changes only which lane
    solves a pair: a six-step graph and three single steps after it give the same states,
    counters and colliding pairs with the order on and off, bit for bit."""
    setup, fn, refs, st = case(name)
    grids = {"gather": 296, "integrate": 592, "bin": 592, "search": 592}
    out = {}
    for on in (False, True):
        with _ctx(setup, fn, st, precision) as ctx:
            ctx.set_launch({**grids, "overlap_gather": True})
            ctx.set_contact_order(on)
            assert ctx.contact_order() == on
            ctx.step(6)
            for _ in range(3):
                ctx.step(1)
            ctx.raise_status()
            out[on] = (ctx.download(), ctx.collision_counters(), ctx.collision_pairs())
    assert out[False][1]["accepted"] > 0
    assert out[True][1] == out[False][1]
    for a, b in zip(out[True][2], out[False][2]):
        assert np.array_equal(a, b)
    for k in api.STATE_KEYS:
        assert np.array_equal(out[True][0][k], out[False][0][k]), k


@pytest.mark.parametrize("name", ["dense", "poly"])
def test_gather_staging_changes_nothing(name):
    """The mixed gather with each particle's stencil box staged in shared memory by the
    TMA (gp_set_gather_staging(1)) sums the same values in the same order as the gather
    of stencil rows through L1: the interpolated fluid values and the states after one
    step and after five more steps with the gather overlapped are the same bit for bit."""
    setup, fn, refs, st = case(name)
    out = {}
    for mode in (0, 1):
        with _ctx(setup, fn, st, "mixed", store_fluid=True) as ctx:
            ctx.set_gather_staging(mode)
            assert ctx.gather_staging() == mode
            ctx.step(1)
            first = ctx.download(fluid=True)
            ctx.set_launch({"gather": 296, "integrate": 592, "bin": 592, "search": 592, "overlap_gather": True})
            assert ctx.gather_staging() == mode
            ctx.step(5)
            ctx.raise_status()
            out[mode] = (first, ctx.download(fluid=True), ctx.collision_counters())
    assert np.all(np.isfinite(out[0][0]["ufap"]))
    for a, b in ((out[0][0], out[1][0]), (out[0][1], out[1][1])):
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    assert out[0][2] == out[1][2]
