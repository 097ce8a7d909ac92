"""Pair buffers sized from counts.

The reference keeps its candidate pairs in a static array of 1e8 entries with no check
(collision.f90:35-37, collision_detection_connectivity.f90:171,189).  Here a step whose
candidates outgrow the buffers stops after its advance, the call that ran it grows the
buffers to the counted need and runs that step's collision phase again, and the
remaining steps follow.  Forcing buffers far too small for the dense case must therefore
give the states and accepted pairs of a run with room from the start, through every
stepping entry point and every overlap choice."""
from __future__ import annotations

import numpy as np
import pytest

from gazpart_b200 import api
from _cases import case

pytestmark = pytest.mark.gpu

GRIDS = {"gather": 296, "integrate": 592, "bin": 592, "search": 592}


def _ctx(setup, fn, st, precision):
    ctx = api.Context(setup, precision)
    ctx.set_fields(fn)
    ctx.upload(st)
    return ctx


def _same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in api.STATE_KEYS)


@pytest.mark.parametrize("overlap", [0, 1, 2])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_small_pair_buffers_grow_and_give_the_same_steps(overlap, precision):
    setup, fn, refs, st = case("dense")
    out = {}
    for small in (False, True):
        with _ctx(setup, fn, st, precision) as ctx:
            ctx.set_launch({**GRIDS, "overlap_gather": overlap > 0, "speculative_integrate": overlap == 2})
            if small:
                ctx.set_pair_capacity(64, 16)
            ctx.step(6)
            ctx.raise_status()
            home, near = ctx.collision_pairs()
            out[small] = (ctx.download(), home, near, ctx.pair_capacity())
    assert _same(out[True][0], out[False][0])
    assert np.array_equal(out[True][1], out[False][1]) and np.array_equal(out[True][2], out[False][2])
    assert out[False][1].size > 0
    cap_pairs, cap_coll = out[True][3]
    assert cap_pairs > 64 and cap_coll > 16


def test_small_pair_buffers_in_collision_and_host_step():
    setup, fn, refs, st = case("dense")
    res = {}
    for small in (False, True):
        with _ctx(setup, fn, st, "fp64") as ctx:
            if small:
                ctx.set_pair_capacity(100, 100)
            cnt = ctx.collision(1, 0.0)
            ctx.raise_status()
            pairs = ctx.collision_pairs()
            after = ctx.download()
            if small:
                ctx.set_pair_capacity(100, 100)
            host = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in after.items()}
            ctx.step_host(host)
            ctx.raise_status()
            res[small] = (cnt, pairs, after, host, ctx.collision_pairs())
    (c0, p0, a0, h0, q0), (c1, p1, a1, h1, q1) = res[False], res[True]
    assert c0["n_coll"] == c1["n_coll"] and c0["n_contact"] == c1["n_contact"]
    assert np.array_equal(p0[0], p1[0]) and np.array_equal(p0[1], p1[1])
    assert _same(a0, a1) and _same(h0, h1)
    assert np.array_equal(q0[0], q1[0]) and np.array_equal(q0[1], q1[1])
    assert p0[0].size > 0
