"""Step parity over a 100-step horizon, with the device re-seeded from the oracle's state
at every step.

Each step n starts both sides from the same state S_n (the oracle's) and checks:

1. ADV_PARTICLE_ELLP (adv_particle_new.f90:7-704): every particle's position, velocity,
   quaternion and angular velocity within 1e-12 relative.  The two sides differ only in
   the libm of the force, torque and quaternion routines (pow, atan, sin, cos from the
   device's math library against the host's), a few ulps.
2. COLLISION (collision.f90:7-200) from the oracle's own post-advance state: every
   particle bit for bit and the accepted pairs identical, in acceptance order.  The
   oracle's pair walk runs without any prefilter (the reference's walk,
   collision_interaction.f90:190-419, one Levenberg-Marquardt solve per candidate pair)
   every tenth step, with the exact prefilters otherwise.
3. The whole step from S_n on the device against the oracle's whole step: accepted pairs
   identical; every particle that took part in no collision within 1e-12.  A particle
   that collided inherits the advance's ulp differences through the contact solve, whose
   stopping point (xtol = sqrt(eps)) moves with its inputs; its error is reported and
   bounded separately.

The bars: integer outputs and pair sets bit-exact, state 1e-12 per
step."""
from __future__ import annotations

import os

import numpy as np
import pytest

import pyoracle as po
from gazpart_b200 import api
from _cases import REL_TOL, case, copy_state, rel_err

pytestmark = pytest.mark.gpu

THREADS = max(1, os.cpu_count() or 1)
# bound on a collided particle's whole-step error (item 3): the LM stopping rule turns
# input differences of a few ulps into contact-point shifts far below xtol = 1.5e-8
COLLIDED_BOUND = 1e-9


def _state(ens):
    return {k: ens.a[k].copy() for k in api.STATE_KEYS}


def _same(a, b, keys):
    return all(np.array_equal(a[k], b[k]) for k in keys)


@pytest.mark.parametrize("name,steps,unfiltered_every", [("poly", 100, 10), ("dense", 100, 10),
                                                          ("bimodal", 100, 1000)])
def test_reseeded_step_parity(name, steps, unfiltered_every):
    setup, fn, refs, st = case(name)
    ens = po.Ensemble(setup, copy_state(st))
    worst_adv = worst_free = worst_coll = 0.0
    n_collided_particles = n_pairs = 0
    with api.Context(setup, "fp64") as ctx:
        ctx.set_fields(fn)
        ctx.upload(st)
        for step in range(steps):
            s0 = _state(ens)
            # 1. the advance from S_n
            ctx.put_state(s0)
            ctx.adv_particle_ellp(step)
            ctx.raise_status(f"advance, step {step}")
            g_adv = ctx.download()
            assert ens.advance(refs, nthreads=THREADS) == 0
            s1 = _state(ens)
            e_adv = rel_err(g_adv, s1, api.STATE_KEYS)
            worst_adv = max(worst_adv, e_adv)
            assert e_adv < REL_TOL, (step, e_adv)
            # 2. the collision phase from the oracle's post-advance state
            ctx.put_state(s1)
            ctx.collision(step, 0.0)
            ctx.raise_status(f"collision, step {step}")
            g_col = ctx.download()
            home, near = ctx.collision_pairs()
            res = ens.collide(prefilter=(step % unfiltered_every != 0), nthreads=THREADS)
            assert res["rc"] == 0
            assert np.array_equal(home, res["home"]) and np.array_equal(near, res["near"]), step
            assert _same(g_col, ens.a, api.STATE_KEYS), step
            # 3. the whole step from S_n
            ctx.put_state(s0)
            ctx.adv_particle_ellp(step)
            ctx.collision(step, 0.0)
            ctx.raise_status(f"step {step}")
            g_full = ctx.download()
            fh, fnr = ctx.collision_pairs()
            assert np.array_equal(fh, res["home"]) and np.array_equal(fnr, res["near"]), step
            hit = np.zeros(ens.n, dtype=bool)
            hit[res["home"]] = True
            hit[res["near"]] = True
            n_collided_particles += int(hit.sum())
            n_pairs += int(res["home"].size)
            free = {k: v[~hit] for k, v in g_full.items()}
            ref_free = {k: ens.a[k][~hit] for k in api.STATE_KEYS}
            e_free = rel_err(free, ref_free, api.STATE_KEYS)
            worst_free = max(worst_free, e_free)
            assert e_free < REL_TOL, (step, e_free)
            if hit.any():
                coll = {k: v[hit] for k, v in g_full.items()}
                ref_coll = {k: ens.a[k][hit] for k in api.STATE_KEYS}
                worst_coll = max(worst_coll, rel_err(coll, ref_coll, api.STATE_KEYS))
    print(f"\n{name}: {steps} steps, {n_pairs} accepted pairs; advance {worst_adv:.2e}, "
          f"collision bit-exact, whole step: free {worst_free:.2e}, collided {worst_coll:.2e} "
          f"over {n_collided_particles} particle-steps")
    assert n_pairs > 0
    assert worst_coll < COLLIDED_BOUND, worst_coll
