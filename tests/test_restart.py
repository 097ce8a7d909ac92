"""Restart files through the device: gp_save_part_class and gp_load_part_class.

A run stopped after some steps, written to a class restart file straight from the
pool and started again from that file in a fresh context, must continue bit for bit
as the run that never stopped; the file's columns must be the state the context
holds, in the class's own particle order."""
from __future__ import annotations

import numpy as np
import pytest

from gazpart_b200 import api, config, field, restart
from _cases import field_refs, init_state

pytestmark = pytest.mark.gpu

SETUP = config.Setup(nx=40, ny=40, nz=40, visc=0.05, dtime=1e-3)


def _steps(ctx, s0, k):
    for s in range(s0, s0 + k):
        ctx.adv_particle_ellp(s)
        ctx.collision(s, 0.0)
    ctx.raise_status()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_restart_continues_bit_for_bit(tmp_path, precision):
    f = field.generate(40, seed=61, device="cpu")
    fn = {k: v.numpy().copy() for k, v in f.items()}
    # one reference-style class: a single shape and density, so the tables hold it
    st = init_state(SETUP, config.ParticleSpec(n=3000, ar=2.5, b=0.03, st=1.0, seed=62), f, field_refs(f))
    assert np.unique(st["emaj"]).size == 1 and np.unique(st["rhop"]).size == 1
    tables = restart.default_tables(3000, st["emaj"][0], st["apr"][0], st["rhop"][0])
    pr = restart.props_from_tables(np.ones(3000, np.int32), tables)
    for k in api.PROP_KEYS:
        assert np.array_equal(pr[k], st[k]), k
    p1 = str(tmp_path / restart.part_file_name(1, 4))
    p2 = str(tmp_path / restart.part_file_name(1, 8))
    with api.Context(SETUP, precision) as a:
        a.set_fields(fn)
        a.upload(st)
        _steps(a, 0, 4)
        restart.save_class(a, 1, p1, tables)
        mid = a.download()
        _steps(a, 4, 4)
        restart.save_class(a, 1, p2, tables)
        end = a.download()
    cols, t1 = restart.read_part_class(p1)
    for k in api.STATE_KEYS:
        assert np.array_equal(cols[k], mid[k]), k
    assert np.all(cols["idp"] == 1) and t1.npclass.tolist() == [3000]
    with api.Context(SETUP, precision, max_particles=3000) as b:
        b.set_fields(fn)
        ig, n = restart.load_class(b, p1)
        assert (ig, n) == (1, 3000)
        _steps(b, 4, 4)
        got = b.download_class(1)
    for k in api.STATE_KEYS:
        assert np.array_equal(got[k], end[k]), k
    cols2, _ = restart.read_part_class(p2)
    for k in api.STATE_KEYS:
        assert np.array_equal(cols2[k], end[k]), k


def test_load_rejects_an_index_outside_the_tables(tmp_path):
    n = 10
    cols = {k: np.zeros(n) for k in restart.PART_COLUMNS}
    cols["qa"][:] = 1.0
    cols["x"][:] = cols["y"][:] = cols["z"][:] = 1.0
    cols["idp"] = np.full(n, 2, np.int32)
    p = str(tmp_path / "part_p01.ini")
    restart.write_part_class(p, cols, restart.default_tables(n, 0.01, 2.0, 1000.0))
    f = field.generate(40, seed=61, device="cpu")
    with api.Context(SETUP, "fp64", max_particles=100) as ctx:
        ctx.set_fields({k: v.numpy().copy() for k, v in f.items()})
        with pytest.raises(api.GPError) as e:
            restart.load_class(ctx, p)
        assert e.value.code == 9           # GP_EBADARG: IDP 2 with one table entry
        assert ctx.n == 0
