"""Several classes stepped together (gp_upload_classes) against each class alone.

Classes never interact: every particle's advance reads only its own record and the
shared field, and collisions are searched, solved and accepted within a class.  So a
class stepped in a batch must end bit for bit where it ends when stepped alone, in both
precision forms, with the same colliding pairs."""
from __future__ import annotations

import numpy as np
import pytest

from gazpart_b200 import api, config, field
from _cases import field_refs, init_state

pytestmark = pytest.mark.gpu

SPECS = [
    config.ParticleSpec(n=600, ar_range=(0.5, 2.0), b=0.03, st=1.0, seed=31),
    config.ParticleSpec(n=5000, ar_range=(0.3, 4.0), b=0.02, st_loguniform=(0.1, 10.0), seed=32),
    config.ParticleSpec(n=12000, ar_range=(1.0, 3.0), b=0.025, st=0.5, seed=33),
    config.ParticleSpec(n=1500, ar_range=(0.2, 5.0), b_lognormal=(np.log(0.01), 0.3), st_uniform=(0.1, 10.0),
                        seed=34),
]


def _inputs():
    setup = config.Setup(nx=48, ny=48, nz=48, visc=0.05, dtime=1e-3)
    f = field.generate(48, seed=17, device="cpu")
    refs = field_refs(f)
    states = [init_state(setup, spec, f, refs) for spec in SPECS]
    return setup, {k: v.numpy().copy() for k, v in f.items()}, states


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_classes_in_one_batch_match_each_class_alone(precision):
    setup, fn, states = _inputs()
    steps = 6
    with api.Context(setup, precision) as batch:
        batch.set_fields(fn)
        batch.upload_classes(states)
        batch.step(steps - 1)
        batch.adv_particle_ellp(steps - 1)
        batch.collision(steps - 1, 0.0)
        batch.raise_status()
        home_b, near_b = batch.collision_pairs()
        got = batch.split_classes(batch.download())
    begin = 0
    total_pairs = 0
    for k, st in enumerate(states):
        with api.Context(setup, precision) as alone:
            alone.set_fields(fn)
            alone.upload(st)
            alone.step(steps - 1)
            alone.adv_particle_ellp(steps - 1)
            alone.collision(steps - 1, 0.0)
            alone.raise_status()
            home_a, near_a = alone.collision_pairs()
            ref = alone.download()
        for key in api.STATE_KEYS:
            assert np.array_equal(got[k][key], ref[key]), (k, key)
        mine = (home_b >= begin) & (home_b < begin + len(st["x"]))
        assert np.array_equal(home_b[mine] - begin, home_a) and np.array_equal(near_b[mine] - begin, near_a)
        total_pairs += home_a.size
        begin += len(st["x"])
    assert home_b.size == total_pairs
    assert total_pairs > 0                      # the classes do collide


def test_autotune_keeps_the_state_and_the_results():
    setup, fn, states = _inputs()
    with api.Context(setup, "fp64") as a, api.Context(setup, "fp64") as b:
        for ctx in (a, b):
            ctx.set_fields(fn)
            ctx.upload_classes(states)
        before = a.download()
        grids = a.autotune()
        a.raise_status()
        after = a.download()
        for key in api.STATE_KEYS:
            assert np.array_equal(before[key], after[key]), key
        assert set(grids) == {"gather", "integrate", "bin", "search", "overlap_gather", "speculative_integrate",
                              "contact_tail", "gather_staging"}
        assert grids["contact_tail"] == 0        # the default; the autotuner leaves it
        assert grids["gather_staging"] == 0      # FP64: rows only
        assert all(grids[k] in (148, 296, 592, 1184, 2368) for k in ("gather", "integrate", "bin", "search"))
        # launch shapes change no result
        a.step(3)
        b.step(3)
        ra, rb = a.download(), b.download()
    for key in api.STATE_KEYS:
        assert np.array_equal(ra[key], rb[key]), key
