"""Serving: jobs streamed into one context with two resident fields (gp_serve).

Jobs arrive while others run, share the same launches, and leave when done.  Each job's
final state must equal, bit for bit, the state of the same job stepped alone in a
context of its own, in both precision forms (the tolerance is zero: a job's arithmetic
does not depend on its neighbours in the pool)."""
from __future__ import annotations

import numpy as np
import pytest

from gazpart_b200 import api, config, field, serving
from _cases import field_refs, init_state

pytestmark = pytest.mark.gpu

PHYS = dict(visc=0.05, dtime=1e-3)


def _fields():
    f0 = field.generate(32, seed=41, device="cpu")
    f1 = field.generate(48, seed=42, device="cpu")
    return [(config.Setup(nx=32, ny=32, nz=32, **PHYS), f0), (config.Setup(nx=48, ny=48, nz=48, **PHYS), f1)]


def _jobs(fields):
    specs = [(0, config.ParticleSpec(n=700, ar_range=(0.5, 2.0), b=0.03, st=1.0, seed=51), 9, 0.0),
             (1, config.ParticleSpec(n=4000, ar_range=(0.3, 4.0), b=0.025, st_loguniform=(0.1, 10.0), seed=52),
              14, 0.0),
             (0, config.ParticleSpec(n=2500, ar=2.0, b=0.02, st=0.5, seed=53, density_from_st=True), 6, 0.03),
             (1, config.ParticleSpec(n=1200, ar_range=(0.2, 5.0), b_lognormal=(np.log(0.01), 0.3),
                                     st_uniform=(0.1, 10.0), seed=54), 11, 0.06),
             (1, config.ParticleSpec(n=300, ar=0.5, b=0.03, st=2.0, seed=55), 0, 0.06)]
    jobs = []
    for fid, spec, steps, t in specs:
        setup, f = fields[fid]
        st = init_state(setup, spec, f, field_refs(f))
        jobs.append(serving.Job(state=st, steps=steps, arrival_s=t, field=fid))
    return jobs


def _alone(setup, f, job, precision):
    with api.Context(setup, precision) as ctx:
        ctx.set_fields({k: v.numpy().copy() for k, v in f.items()})
        ctx.upload({k: np.array(v, copy=True) for k, v in job.state.items()})
        for s in range(job.steps):
            ctx.adv_particle_ellp(s)
            ctx.collision(s, 0.0)
        ctx.raise_status()
        return ctx.download()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_each_job_in_the_mix_matches_the_job_alone(precision):
    fields = _fields()
    jobs = _jobs(fields)
    (s0, f0), (s1, f1) = fields
    with api.Context(s0, precision, max_particles=20000) as ctx:
        ctx.set_fields({k: v.numpy().copy() for k, v in f0.items()})
        fid = ctx.add_field(48)
        assert fid == 1
        ctx.set_fields({k: v.numpy().copy() for k, v in f1.items()}, slot=1)
        summary = serving.serve(ctx, jobs, hbm_budget=1e9)
    assert summary["failed"] == 0
    assert summary["particle_steps"] == sum(j.n * j.steps for j in jobs)
    assert summary["max_concurrent"] >= 2            # their work shared launches
    for j in jobs:
        assert j.arrival_s <= j.admitted_s <= j.done_s
        setup, f = fields[j.field]
        ref = _alone(setup, f, j, precision)
        for k in api.STATE_KEYS:
            assert np.array_equal(j.result[k], ref[k]), (j.field, j.n, k)


def test_admission_waits_for_the_budget():
    fields = _fields()
    jobs = [_jobs(fields)[i] for i in (0, 2, 3)]      # 700, 2500 and 1200 particles
    for j in jobs:
        j.arrival_s = 0.0
    s0, f0 = fields[0]
    with api.Context(s0, "fp64", max_particles=20000) as ctx:
        ctx.set_fields({k: v.numpy().copy() for k, v in f0.items()})
        ctx.add_field(48)
        ctx.set_fields({k: v.numpy().copy() for k, v in fields[1][1].items()}, slot=1)
        # no two of them fit together: first come first served, one after another
        budget = 2600 * serving.BYTES_PER_PARTICLE
        summary = serving.serve(ctx, jobs, hbm_budget=budget)
    assert summary["failed"] == 0 and summary["max_concurrent"] == 1
    order = sorted(jobs, key=lambda j: j.admitted_s)
    for a, b in zip(order, order[1:]):
        assert a.done_s <= b.admitted_s
