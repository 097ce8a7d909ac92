"""Wall-bounded channel mode (FROZEN_FLOW = 3, WALL_BOUNDARY = .true.).

The channel keeps the step of the periodic box with three differences: the stencil
mirrors at the walls x = 0 and x = L instead of wrapping (interp_lag3.f90:132-154),
the box grid and the minimum image do not wrap in x (PERIODICITY = .false.), and after
the advance only y and z wrap (BOUNDARY_PARTICLE_Y_Z, adv_particle_new.f90:685).  The
field is the mean-profile channel of initiation_frozen_flow.f90:77-155.  The profile
used here is a test input of its own (a parabola), not one of the reference's files,
which it does not ship."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle as po
from gazpart_b200 import api, config, field, particles
from _cases import REL_TOL, rel_err

L = 2.0 * np.pi
N_IN = field.CHANNEL_POINTS


def _profile():
    x_in = L / (N_IN - 1) * np.arange(N_IN)
    ug = 1.0 - (2.0 * x_in / L - 1.0) ** 2
    vorty = 4.0 / L * (2.0 * x_in / L - 1.0)
    return x_in, ug, vorty


def _setup(n=41):
    return config.Setup(nx=n, ny=n, nz=n, visc=0.05, dtime=1e-3, periodicity=False, wall_boundary=True,
                        frozen_flow=3)


def test_channel_field_from_profiles(tmp_path):
    x_in, ug, vorty = _profile()
    up, vp = tmp_path / "Ug_mean.in", tmp_path / "vorticity_y.txt"
    up.write_text("".join(f"{float(a)!r}   {float(b)!r}\n" for a, b in zip(x_in, ug)))
    vp.write_text("".join(f"  {float(c)!r}\n" for c in vorty))
    xr, ur, vr = field.read_channel_profiles(str(up), str(vp))
    assert np.array_equal(xr, x_in) and np.array_equal(ur, ug) and np.array_equal(vr, vorty)
    s = _setup()
    f = field.channel(s, xr, ur, vr, po.frozen_interp_lag3)
    w = f["w"].numpy()
    assert w.shape == (41, 41, 41)
    assert np.all(w == w[:1, :1, :])                       # W varies along x only
    xm = s.dx * np.arange(41)
    # exact on a parabola where the cubic stencil stays inside the 21 points; in the end
    # intervals FROZEN_INTERP_LAG3 mirrors the stencil (frozen_interp_lag3.f90:130-158)
    assert np.max(np.abs(w[0, 0, 4:-4] - (1.0 - (2.0 * xm[4:-4] / L - 1.0) ** 2))) < 1e-12
    assert np.array_equal(w[0, 0, ::2], ug)                 # the profile's own nodes
    vy = f["vorty"].numpy()
    assert np.all(vy == vy[:1, :, :1])                      # the vorticity profile lies along y
    assert np.max(np.abs(vy[0, 4:-4, 0] - 4.0 / L * (2.0 * xm[4:-4] / L - 1.0))) < 1e-12
    for k in ("u", "v", "vortx", "vortz"):
        assert not f[k].any()
    with pytest.raises(ValueError):
        field.channel(config.Setup(nx=41, ny=33, nz=41, wall_boundary=True, periodicity=False, frozen_flow=3),
                      xr, ur, vr, po.frozen_interp_lag3)


def _channel_state(s, f):
    """Spheroids in the channel, some heading for the walls, some about to cross z = L."""
    refs = [field.reference_layout(f[k], "periodic" if k in ("u", "v", "w") else "zero").numpy().copy()
            for k in field.COMPONENTS_6]
    spec = config.ParticleSpec(n=4000, ar_range=(0.8, 1.5), b=0.02, st=1.0, seed=71)
    st = particles.draw(spec, s)
    uf = [po.interp_lag3(s, refs[c], st["x"], st["y"], st["z"]) for c in range(6)]
    st["u"], st["v"], st["w"] = uf[0].copy(), uf[1].copy(), uf[2].copy()
    particles.body_half_vorticity(st, uf[3], uf[4], uf[5])
    # x extent of each spheroid: sqrt(b^2 + (a^2 - b^2) e_x^2), e = R(q) (1,0,0)
    a_, b_ = st["emaj"], st["emaj"] / st["apr"]
    ex = 1.0 - 2.0 * (st["qc"] ** 2 + st["qd"] ** 2)
    hx = np.sqrt(b_ * b_ + (a_ * a_ - b_ * b_) * ex * ex)
    k = np.arange(40)
    st["x"][k] = np.where(k % 2 == 0, hx[k] + 0.002, L - hx[k] - 0.002)   # near a wall, closing on it
    st["u"][k] = np.where(k % 2 == 0, -0.8, 0.8)
    j = np.arange(40, 60)
    st["z"][j] = L - 0.001
    st["w"][j] = 0.5                                                     # crosses z = L
    st["y"][j] = 0.001
    st["v"][j] = -0.5                                                    # crosses y = 0
    return st, refs


@pytest.mark.gpu
def test_channel_steps_match_oracle():
    s = _setup()
    x_in, ug, vorty = _profile()
    with api.Context(s, "fp64") as probe:
        dev_field = field.channel(s, x_in, ug, vorty, probe.frozen_interp_lag3)
    f = field.channel(s, x_in, ug, vorty, po.frozen_interp_lag3)
    for k in field.COMPONENTS_6:
        assert np.array_equal(dev_field[k].numpy(), f[k].numpy()), k
    fn = {k: v.numpy().copy() for k, v in f.items()}
    st, refs = _channel_state(s, f)
    ens = po.Ensemble(s, {k: np.array(v, copy=True) for k, v in st.items()})
    collided = np.zeros(ens.n, dtype=bool)
    x0 = st["x"].copy()
    with api.Context(s, "fp64") as ctx:
        ctx.set_fields(fn)
        ctx.upload(st)
        for step in range(12):
            assert ens.advance(refs, nthreads=8) == 0
            res = ens.collide(prefilter=True, nthreads=8)
            assert res["rc"] == 0
            collided[res["home"]] = True
            collided[res["near"]] = True
            ctx.adv_particle_ellp(step)
            ctx.collision(step, 0.0)
            if step == 0:
                home, near = ctx.collision_pairs()
                assert np.array_equal(home, res["home"]) and np.array_equal(near, res["near"])
        ctx.raise_status()
        got = ctx.download()
    free = {k: v[~collided] for k, v in got.items()}
    assert rel_err(free, {k: ens.a[k][~collided] for k in api.STATE_KEYS}, api.STATE_KEYS) < REL_TOL
    assert rel_err(got, ens.a, api.STATE_KEYS) < 1e-9
    k = np.arange(40)
    assert np.all(np.sign(got["u"][k]) == np.where(k % 2 == 0, 1.0, -1.0))   # rebounded off the walls
    assert np.all((got["x"] > 0.0) & (got["x"] < L))                           # x never wraps
    j = np.arange(40, 60)
    assert np.all(got["z"][j] < 0.01) and np.all(got["y"][j] > L - 0.01)      # y and z wrapped
    assert np.any(got["x"] != x0)


@pytest.mark.gpu
def test_channel_mixed_gather_staging_changes_nothing():
    """In the channel the stencils next to the walls are mirrored (not four contiguous
    points), and the TMA-staged mixed gather leaves those to per-lane loads: six steps
    give the row gather's states and fluid values bit for bit."""
    s = _setup()
    x_in, ug, vorty = _profile()
    f = field.channel(s, x_in, ug, vorty, po.frozen_interp_lag3)
    fn = {k: v.numpy().copy() for k, v in f.items()}
    st, refs = _channel_state(s, f)
    out = {}
    for mode in (0, 1):
        with api.Context(s, "mixed", store_fluid=True) as ctx:
            ctx.set_fields(fn)
            ctx.upload(st)
            ctx.set_gather_staging(mode)
            assert ctx.gather_staging() == mode
            ctx.step(6)
            ctx.raise_status()
            out[mode] = ctx.download(fluid=True)
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k], equal_nan=True), k
