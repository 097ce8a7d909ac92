"""The live-fluid step (ADV_FLUID) on the device against the numpy restatement.

CPU tests pin the restatement (oracle/spectral.py) on known answers; GPU tests hold the
device solver (gp_dns_*) to it.  The two run different FFT implementations (cuFFT and
numpy's pocketfft), whose results differ in the last bits, so the fields are compared
to 1e-12 of their magnitude per step, and a particle run coupled to the live field to
1e-10 over a few cycles."""
from __future__ import annotations

import numpy as np
import pytest
import torch

import spectral
import pyoracle as po
from gazpart_b200 import api, config, field, particles
from _cases import rel_err

L = 2.0 * np.pi


def _shear(n, amp=0.3, k=2):
    z, y, x = np.meshgrid(*(np.arange(n) * (L / n) for _ in range(3)), indexing="ij")
    u = amp * np.sin(k * y)
    return u, np.zeros_like(u), np.zeros_like(u)


def test_shear_wave_decays_by_the_integrating_factor():
    """u = A sin(k y) x: u x omega is a gradient, so the projected nonlinear term
    vanishes and each step multiplies the mode by exp(-visc k^2 dt)."""
    n, visc, dt = 16, 0.05, 0.01
    sp = spectral.Spectral(n, n, n, L, visc, dt)
    u, v, w = _shear(n)
    u0 = u.copy()
    for _ in range(10):
        u, v, w = sp.adv_fluid(u, v, w)
    assert np.max(np.abs(u - u0 * np.exp(-visc * 4 * 10 * dt))) < 1e-13
    assert np.max(np.abs(v)) < 1e-14 and np.max(np.abs(w)) < 1e-14


def test_taylor_green_decay_and_divergence():
    """A weak Taylor-Green vortex decays at the viscous rate 2 visc k^2 (k^2 = 3) to
    within its amplitude squared; every step leaves the field divergence-free."""
    n, visc, dt, amp = 16, 0.1, 0.01, 1e-3
    sp = spectral.Spectral(n, n, n, L, visc, dt)
    z, y, x = np.meshgrid(*(np.arange(n) * (L / n) for _ in range(3)), indexing="ij")
    u = amp * np.sin(x) * np.cos(y) * np.cos(z)
    v = -amp * np.cos(x) * np.sin(y) * np.cos(z)
    w = np.zeros_like(u)
    e0 = np.mean(u * u + v * v)
    for _ in range(20):
        u, v, w = sp.adv_fluid(u, v, w)
        assert np.max(np.abs(sp.divergence_hat(u, v, w))) < 1e-12 * amp * n ** 3
    e = np.mean(u * u + v * v + w * w)
    assert abs(e / e0 - np.exp(-2 * visc * 3 * 20 * dt)) < 10 * amp


def test_vorticity_of_a_shear():
    n = 16
    sp = spectral.Spectral(n, n, n, L, 0.05, 0.01)
    u, v, w = _shear(n, amp=0.5, k=3)
    ox, oy, oz = sp.vorticity(u, v, w)
    z, y, x = np.meshgrid(*(np.arange(n) * (L / n) for _ in range(3)), indexing="ij")
    assert np.max(np.abs(oz + 0.5 * 3 * np.cos(3 * y))) < 1e-13        # omega_z = -du/dy
    assert np.max(np.abs(ox)) < 1e-14 and np.max(np.abs(oy)) < 1e-14


def _random_field(n, seed):
    f = field.generate(n, lbox=L, seed=seed, device="cpu")
    return [f[k].numpy().copy() for k in ("u", "v", "w")]


@pytest.mark.gpu
def test_adv_fluid_matches_restatement():
    from gazpart_b200 import dns
    n = 32
    s = config.Setup(nx=n, ny=n, nz=n, visc=0.02, dtime=0.005)
    sp = spectral.Spectral(n, n, n, s.lx, s.visc, s.dtime)
    u, v, w = _random_field(n, 81)
    with dns.Fluid(s) as fl:
        fl.set_velocity(u, v, w)
        ref = (u, v, w)
        for step in range(5):
            fl.adv_fluid(step)
            ref = sp.adv_fluid(*ref)
            got = fl.velocity()
            scale = max(np.max(np.abs(r)) for r in ref)
            err = max(np.max(np.abs(g - r)) for g, r in zip(got, ref))
            assert err < 1e-12 * scale * (step + 1), (step, err / scale)
        vort = fl.vorticity()
    for g, r in zip(vort, sp.vorticity(*ref)):
        assert np.max(np.abs(g - r)) < 1e-12 * np.max(np.abs(r))


@pytest.mark.gpu
def test_particles_follow_the_live_field():
    """Each cycle as main.f90 orders it: the particles step through the current field,
    then ADV_FLUID, then the field refresh.  The vorticity stays as set at the start,
    as the reference's arrays do in DNS mode."""
    from gazpart_b200 import dns
    n = 32
    s = config.Setup(nx=n, ny=n, nz=n, visc=0.02, dtime=0.005)
    sp = spectral.Spectral(n, n, n, s.lx, s.visc, s.dtime)
    f = field.generate(n, lbox=s.lx, seed=83, device="cpu")
    fn = {k: v.numpy().copy() for k, v in f.items()}
    refs = [field.reference_layout(f[k], "periodic" if k in ("u", "v", "w") else "zero").numpy().copy()
            for k in field.COMPONENTS_6]
    st = particles.draw(config.ParticleSpec(n=2000, ar_range=(0.5, 2.0), b=0.02, st=1.0, seed=84), s)
    uf = [po.interp_lag3(s, refs[c], st["x"], st["y"], st["z"]) for c in range(6)]
    st["u"], st["v"], st["w"] = uf[0].copy(), uf[1].copy(), uf[2].copy()
    particles.body_half_vorticity(st, uf[3], uf[4], uf[5])
    ens = po.Ensemble(s, {k: np.array(v, copy=True) for k, v in st.items()})
    vel = [fn["u"], fn["v"], fn["w"]]
    with api.Context(s, "fp64") as ctx, dns.Fluid(s) as fl:
        ctx.set_fields(fn)
        ctx.upload(st)
        fl.set_velocity(*vel)
        for cyc in range(4):
            assert ens.advance(refs, nthreads=8) == 0
            assert ens.collide(prefilter=True, nthreads=8)["rc"] == 0
            ctx.adv_particle_ellp(cyc)
            ctx.collision(cyc, 0.0)
            vel = list(sp.adv_fluid(*vel))
            for c in range(3):
                refs[c] = field.reference_layout(torch.from_numpy(vel[c]), "periodic").numpy().copy()
            fl.adv_fluid(cyc)
            fl.couple(ctx)
        ctx.raise_status()
        got = ctx.download()
    assert rel_err(got, ens.a, api.STATE_KEYS) < 1e-10


@pytest.mark.gpu
def test_coupling_refuses_another_mesh():
    from gazpart_b200 import dns
    s32 = config.Setup(nx=32, ny=32, nz=32, visc=0.02, dtime=0.005)
    s16 = config.Setup(nx=16, ny=16, nz=16, visc=0.02, dtime=0.005)
    with api.Context(s16, "fp64") as ctx, dns.Fluid(s32) as fl:
        with pytest.raises(api.GPError) as e:
            fl.couple(ctx)
        assert e.value.code == 9                        # GP_EBADARG: the meshes differ
