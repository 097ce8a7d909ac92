"""Statistics beside the step on the device against the oracle.

STAT_PARTFLUID: the device sums each of the 35 quantities per polydisperse index over
the class's particles.  The oracle sums the same quantities in particle order from
the per-particle shape and density, while the device recovers APR, PMASS and RHOP from
the pool's derived constants to a few units in the last place, and FP64 pow/atan/log
differ in the last place between the device and the host.  So each sum must agree to
1e-11 of the sum of the magnitudes of its terms (NaN where the reference's arithmetic
gives NaN, as for TAUPF of an oblate particle), and the counts exactly.

Collision statistics: the same pre-collision state, one collision step.  The counts of
contacts examined by the COLOR walk and of collisions must agree exactly, the sums of
depth, NVREL, |v_rel| and angle to 1e-9 of the sums of magnitudes (the contact points
come from the same Levenberg-Marquardt iterates, with last-place differences in sin and
cos)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import pyoracle as po
from gazpart_b200 import api
from _cases import case, copy_state

pytestmark = pytest.mark.gpu


def _per_particle(ens, setup):
    """[n, 36] per-particle STAT_PARTFLUID quantities from the oracle."""
    s = po.make_setup(setup)
    out = np.zeros((ens.n, 36))
    a = ens.a
    for i in range(ens.n):
        v = np.zeros(36)
        po.lib().orc_stat_partfluid_particle(
            C.byref(s), C.c_double(a["emaj"][i]), C.c_double(a["apr"][i]), C.c_double(a["rhop"][i]),
            po.dptr(np.array([a["u"][i], a["v"][i], a["w"][i]])), po.dptr(np.array([a["ox"][i], a["oy"][i], a["oz"][i]])),
            po.dptr(np.array([a["qa"][i], a["qb"][i], a["qc"][i], a["qd"][i]])),
            po.dptr(np.array([a["ufap"][i], a["vfap"][i], a["wfap"][i]])),
            po.dptr(np.array([a["vortx"][i], a["vorty"][i], a["vortz"][i]])), po.dptr(v))
        out[i] = v
    return out


@pytest.mark.parametrize("name", ["c1", "poly"])
def test_stat_partfluid_matches_oracle(name):
    setup, fn, refs, st = case(name)
    n = st["x"].size
    idp = (np.arange(n) % 3 + 1).astype(np.int32)
    with api.Context(setup, "fp64", store_fluid=True) as ctx:
        ctx.set_fields(fn)
        ctx.upload(st)
        with pytest.raises(api.GPError):
            ctx.stat_partfluid(1)                 # no step has sampled the fluid yet
        ctx.set_class_groups(1, idp)
        for s in range(3):
            ctx.adv_particle_ellp(s)
            ctx.collision(s, 0.0)
        ctx.step(1)
        ctx.put_state(ctx.download())       # a new state: no fluid sample for it ...
        with pytest.raises(api.GPError):
            ctx.stat_partfluid(1)
        ctx.step(1)                         # ... until a step, here a graph replay, takes one
        ctx.raise_status()
        sums = ctx.stat_partfluid(1, sums=True)
        means = ctx.stat_partfluid(1)
        got = ctx.download(fluid=True)
    ens = po.Ensemble(setup, {k: got[k] for k in api.STATE_KEYS} | {k: st[k] for k in api.PROP_KEYS})
    for k in api.FLUID_KEYS:
        ens.a[k] = np.ascontiguousarray(got[k])
    ref = ens.stat_partfluid(idp, 3)
    per = _per_particle(ens, setup)
    assert sums.shape == (3, 36)
    for g in range(3):
        mag = np.abs(per[idp == g + 1]).sum(axis=0)
        nan_ref = np.isnan(ref[g])
        assert np.array_equal(np.isnan(sums[g]), nan_ref), g
        ok = ~nan_ref
        assert np.all(np.abs(sums[g][ok] - ref[g][ok]) <= 1e-11 * mag[ok] + 1e-300), (g, np.flatnonzero(
            np.abs(sums[g][ok] - ref[g][ok]) > 1e-11 * mag[ok]))
        assert sums[g, 35] == np.count_nonzero(idp == g + 1)
        assert means[g, 35] == sums[g, 35]
        assert np.allclose(means[g, :35][ok[:35]], (sums[g, :35] / sums[g, 35])[ok[:35]], rtol=0, atol=0)


@pytest.mark.parametrize("name", ["dense", "poly"])
def test_collision_stats_match_oracle(name):
    setup, fn, refs, st = case(name)
    n = st["x"].size
    idp = (np.arange(n) % 2 + 1).astype(np.int32)
    rc, ref, ncoll = po.Ensemble(setup, copy_state(st)).collide_stats(idp, 2)
    assert rc == 0
    with api.Context(setup, "fp64") as ctx:
        ctx.set_fields(fn)
        ctx.upload(st)
        ctx.set_class_groups(1, idp)
        ctx.enable_collision_stats(True)
        ctx.collision(1, 0.0)
        ctx.raise_status()
        got, steps = ctx.collision_stats(1)
        home, near = ctx.collision_pairs()
    assert steps == 1 and home.size == ncoll
    assert got.shape == (2, 2, 8)
    assert ref[:, :, 0].sum() > 0 and ref[:, :, 1].sum() > 0          # contacts and collisions happen
    assert np.array_equal(got[:, :, 0], ref[:, :, 0])                  # contacts the walk examines
    assert np.array_equal(got[:, :, 1], ref[:, :, 1])                  # collisions
    assert np.array_equal(got[:, :, 2], ref[:, :, 2])
    for k in (3, 5, 6, 7):
        scale = np.abs(ref[:, :, k]) + 1e-300
        if k == 5:
            scale = ref[:, :, 6] + 1e-300                              # |NVREL| <= |v_rel|
        if k == 7:
            scale = ref[:, :, 0] * np.pi + 1e-300
        assert np.all(np.abs(got[:, :, k] - ref[:, :, k]) <= 1e-9 * scale), (k, got[:, :, k], ref[:, :, k])


def test_collision_stats_accumulate_over_graph_steps():
    setup, fn, refs, st = case("dense")
    with api.Context(setup, "fp64") as ctx:
        ctx.set_fields(fn)
        ctx.upload(st)
        ctx.step(1)
        ctx.enable_collision_stats(True)
        ctx.step(3)
        ctx.raise_status()
        acc, steps = ctx.collision_stats(1, reset=False)
        assert steps == 3 and acc[0, 0, 0] > 0
        again, steps2 = ctx.collision_stats(1)          # same sums, then cleared
        assert steps2 == 3 and np.array_equal(np.nan_to_num(again), np.nan_to_num(acc))
        cleared, steps3 = ctx.collision_stats(1)
        assert steps3 == 0 and cleared[0, 0, 0] == 0
        ctx.enable_collision_stats(False)
        ctx.step(2)
        none, steps4 = ctx.collision_stats(1)
        assert steps4 == 0 and none[0, 0, 0] == 0
