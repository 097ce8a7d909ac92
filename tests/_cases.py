"""Seeded parity cases shared by the tests (small enough for the oracle)."""
from __future__ import annotations

import functools

import numpy as np

import pyoracle as po
from gazpart_b200 import config, field, particles

REL_TOL = 1e-12   # FP64 state tolerance per step over the 100-step horizon


def field_refs(f):
    return [field.reference_layout(f[k], "periodic" if k in ("u", "v", "w") else "zero").numpy().copy()
            for k in field.COMPONENTS_6]


def init_state(setup, spec, f, refs):
    st = particles.draw(spec, setup)
    uf = [po.interp_lag3(setup, refs[c], st["x"], st["y"], st["z"]) for c in range(6)]
    st["u"], st["v"], st["w"] = uf[0].copy(), uf[1].copy(), uf[2].copy()
    particles.body_half_vorticity(st, uf[3], uf[4], uf[5])
    return st


@functools.lru_cache(maxsize=None)
def case(name: str):
    """(setup, field dict (numpy), reference-layout fields, initial state)."""
    if name == "c1":
        w = config.C1
        setup = w.setup()
        f = field.generate(w.grid, seed=w.field_seed, device="cpu")
        spec = w.spec
    elif name == "dense":
        # many overlapping spheroids: stresses contacts and the greedy acceptance order
        setup = config.Setup(nx=48, ny=48, nz=48, visc=0.05, dtime=1e-3)
        f = field.generate(48, seed=5, device="cpu")
        spec = config.ParticleSpec(n=20000, ar_range=(0.4, 3.0), b=0.03, st=1.0, seed=11)
    elif name == "poly":
        # polydisperse oblate + prolate, per-particle densities
        setup = config.Setup(nx=48, ny=48, nz=48, visc=0.02, dtime=5e-4)
        f = field.generate(48, seed=9, device="cpu")
        spec = config.ParticleSpec(n=8000, ar_range=(0.2, 5.0), b_lognormal=(np.log(0.01), 0.3),
                                   st_uniform=(0.1, 10.0), seed=4)
    elif name == "bimodal":
        # 20000 small spheroids and a dozen large ones (0.06%): the large ones exceed the
        # search grid's one-cell reach and take the wide-stencil path
        setup = config.Setup(nx=48, ny=48, nz=48, visc=0.05, dtime=1e-3)
        f = field.generate(48, seed=13, device="cpu")
        spec = config.ParticleSpec(n=20000, ar_range=(0.5, 2.0), b=0.02, st=1.0, seed=21)
        big = config.ParticleSpec(n=12, ar_range=(0.4, 3.0), b=0.08, st=1.0, seed=22)
    elif name == "bimodal_small":
        # the bimodal mix at a fifth of the small particles: cheap enough for the oracle's
        # unfiltered pair walk in the CPU suite
        setup = config.Setup(nx=48, ny=48, nz=48, visc=0.05, dtime=1e-3)
        f = field.generate(48, seed=13, device="cpu")
        spec = config.ParticleSpec(n=4000, ar_range=(0.5, 2.0), b=0.03, st=1.0, seed=23)
        big = config.ParticleSpec(n=6, ar_range=(0.4, 3.0), b=0.08, st=1.0, seed=24)
    else:
        raise KeyError(name)
    fn = {k: v.numpy().copy() for k, v in f.items()}
    refs = field_refs(f)
    st = init_state(setup, spec, f, refs)
    if name in ("bimodal", "bimodal_small"):
        st_big = init_state(setup, big, f, refs)
        st = {k: np.concatenate([st[k], st_big[k]]) for k in st}
    return setup, fn, refs, st


def copy_state(st):
    return {k: np.array(v, copy=True) for k, v in st.items()}


def rel_err(a: dict, b: dict, keys) -> float:
    """max over particles of |a-b| / (|b| + 1e-30), vector-wise per group."""
    groups = {"x": ("x", "y", "z"), "u": ("u", "v", "w"), "q": ("qa", "qb", "qc", "qd"), "o": ("ox", "oy", "oz")}
    worst = 0.0
    for g, ks in groups.items():
        if not set(ks) <= set(keys):
            continue
        da = np.sqrt(sum((a[k] - b[k]) ** 2 for k in ks))
        nb = np.sqrt(sum(b[k] ** 2 for k in ks))
        worst = max(worst, float(np.max(da / (nb + 1e-30))))
    return worst
