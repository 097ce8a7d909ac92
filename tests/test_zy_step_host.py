"""gp_step_host: one step of a host-resident ensemble in one call, with the copies
overlapped with the step, against gp_put_state, gp_step(ctx, 1) and gp_download_state
in turn.  The kernels and their order are the same, so the states must agree bit for
bit, step after step."""
from __future__ import annotations

import numpy as np
import pytest

from gazpart_b200 import api
from _cases import case

pytestmark = pytest.mark.gpu


def _ctx(setup, fn, st, precision):
    ctx = api.Context(setup, precision)
    ctx.set_fields(fn)
    ctx.upload(st)
    return ctx


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_host_equals_put_step_download(precision):
    setup, fn, refs, st = case("dense")
    ref = {k: np.array(st[k], dtype=np.float64, copy=True) for k in api.STATE_KEYS}
    got = {k: v.copy() for k, v in ref.items()}
    sep_in = {k: v.copy() for k, v in ref.items()}
    sep_out = {k: np.zeros_like(v) for k, v in ref.items()}
    with _ctx(setup, fn, st, precision) as a, _ctx(setup, fn, st, precision) as b, \
            _ctx(setup, fn, st, precision) as c:
        for _ in range(3):
            a.put_state(ref)
            a.step(1)
            a.download_into(ref)
            b.step_host(got)                        # the same arrays in and out
            c.step_host(sep_in, sep_out)            # separate arrays
            for k in api.STATE_KEYS:
                sep_in[k][:] = sep_out[k]
        a.raise_status()
        b.raise_status()
        c.raise_status()
        assert b.collision_counters() == a.collision_counters()
    for k in api.STATE_KEYS:
        assert np.array_equal(got[k], ref[k]), k
        assert np.array_equal(sep_out[k], ref[k]), k


def test_step_host_rejects_bad_arrays():
    setup, fn, refs, st = case("dense")
    with _ctx(setup, fn, st, "fp64") as a:
        bad = {k: np.array(st[k], dtype=np.float64, copy=True) for k in api.STATE_KEYS}
        bad["x"] = bad["x"][:-1].copy()
        with pytest.raises(ValueError):
            a.step_host(bad)
