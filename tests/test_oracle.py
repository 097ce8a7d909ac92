"""The oracle against known answers, invariants and golden MINPACK vectors.

The reference ships no tests or fixtures; these pin the restatement instead (analytic
results of the algebra it implements, the reference's own runtime invariants, and
scipy's MINPACK for the vendored Levenberg-Marquardt solver).
"""
from __future__ import annotations

import ctypes as C
import itertools
import json
import os

import numpy as np
import pytest

import pyoracle as po
from gazpart_b200 import config, field, particles

HERE = os.path.dirname(os.path.abspath(__file__))


def _setup(n=32, **kw):
    return config.Setup(nx=n, ny=n, nz=n, **kw)


def _unit_q(rng):
    q = rng.normal(size=4)
    return q / np.linalg.norm(q)


# -- interpolation -------------------------------------------------------------
def test_interp_reproduces_cubics_away_from_wrap():
    s = _setup(24)
    rng = np.random.default_rng(0)
    c = rng.normal(size=(4, 4, 4))
    def poly(x, y, z):
        return sum(c[i, j, k] * x ** i * y ** j * z ** k for i in range(4) for j in range(4) for k in range(4))
    i = np.arange(s.nx) * s.dx
    zz, yy, xx = np.meshgrid(i, i, i, indexing="ij")
    import torch
    f = field.reference_layout(torch.from_numpy(poly(xx / 6, yy / 6, zz / 6)), "periodic").numpy().copy()
    pts = rng.uniform(2 * s.dx, s.lx - 3 * s.dx, size=(3, 500))
    got = po.interp_lag3(s, f, *pts)
    ref = poly(*(pts / 6))
    assert np.max(np.abs(got - ref)) < 1e-10 * np.max(np.abs(ref))


def test_interp_at_nodes_is_exact():
    s = _setup(16)
    rng = np.random.default_rng(1)
    import torch
    inner = rng.normal(size=(16, 16, 16))
    f = field.reference_layout(torch.from_numpy(inner), "periodic").numpy().copy()
    idx = rng.integers(0, 15, size=(3, 100))
    got = po.interp_lag3(s, f, idx[0] * s.dx, idx[1] * s.dy, idx[2] * s.dz)
    assert np.allclose(got, inner[idx[2], idx[1], idx[0]], rtol=0, atol=1e-13)


def test_frozen_interp_mirror_matches_interior():
    rng = np.random.default_rng(2)
    n = 12
    u = rng.normal(size=(n, n, n))
    ax = np.arange(n) * 0.1
    pts = rng.uniform(0.25, 0.8, size=(3, 50))
    got = po.frozen_interp_lag3(ax, ax, ax, u, *pts)
    s = config.Setup(nx=n, ny=n, nz=n, lx=0.1 * (n - 1), ly=0.1 * (n - 1), lz=0.1 * (n - 1))
    import torch
    ref = po.interp_lag3(s, field.reference_layout(torch.from_numpy(u), "periodic").numpy().copy(), *pts)
    assert np.allclose(got, ref, atol=1e-12)


# -- rotations -----------------------------------------------------------------
def test_transform_is_quaternion_rotation():
    rng = np.random.default_rng(3)
    for _ in range(20):
        q, v = _unit_q(rng), rng.normal(size=3)
        qv = np.array([0.0, *v])
        def mul(a, b):
            return np.array([a[0] * b[0] - a[1:] @ b[1:], *(a[0] * b[1:] + b[0] * a[1:] + np.cross(a[1:], b[1:]))])
        ref = mul(mul(q, qv), q * [1, -1, -1, -1])[1:]
        assert np.allclose(po.transform_vec(v, q), ref, atol=1e-14)


def test_quaternion_integration_constant_spin():
    rng = np.random.default_rng(4)
    q = _unit_q(rng)
    om = rng.normal(size=3)   # body frame
    dt = 1e-3
    q1 = po.quaternion_integration(q, om, dt)
    w = po.transform_vec(om, q)   # lab frame
    th = np.linalg.norm(w) * dt
    e = np.array([np.cos(th / 2), *(np.sin(th / 2) * w / np.linalg.norm(w))])
    ref = np.array([e[0] * q[0] - e[1:] @ q[1:], *(e[0] * q[1:] + q[0] * e[1:] + np.cross(e[1:], q[1:]))])
    assert np.allclose(q1, ref, atol=1e-15)
    assert abs(np.linalg.norm(q1) - 1) < 1e-15
    # zero spin leaves q unchanged
    assert np.array_equal(po.quaternion_integration(q, [0, 0, 0], dt), q)


def test_euler_integration_conserves_energy_and_momentum():
    ip = (0.4, 1.0, 1.0)
    om = np.array([0.3, 2.0, -1.0])
    E0 = 0.5 * np.dot(ip, om ** 2)
    L0 = np.linalg.norm(np.array(ip) * om)
    for _ in range(100):
        om = po.euler_integration(ip, om, 1e-3)
    assert abs(0.5 * np.dot(ip, om ** 2) - E0) < 1e-10 * E0
    assert abs(np.linalg.norm(np.array(ip) * om) - L0) < 1e-10 * L0


# -- force / torque --------------------------------------------------------------
def test_force_guard_and_drag_direction():
    s = _setup(visc=0.01)
    q = np.array([1.0, 0, 0, 0])
    rc, fd, fl = po.fluid_force(s, 0.01, 2.0, 1000.0, [0.5, 0.5, 0.5], [0.5, 0.5, 0.5], q)
    assert rc == 0 and not fd.any() and not fl.any()
    rc, fd, fl = po.fluid_force(s, 0.01, 2.0, 1000.0, [0, 0, 0], [0.3, 0.0, 0.0], q)
    assert rc == 0 and fd[0] > 0 and abs(fd[1]) == 0 and abs(fl[1]) == 0   # axial flow: no lift


def test_torque_zero_relative_spin_is_zero():
    s = _setup(visc=0.01)
    rng = np.random.default_rng(5)
    q = _unit_q(rng)
    vort = rng.normal(size=3)
    om = 0.5 * po.transform_vec(vort, q * [1, -1, -1, -1])
    rc, tp, tr = po.fluid_torque(s, 0.01, 3.0, 1000.0, [0, 0, 0], [0, 0, 0], vort, om, q)
    assert rc == 0 and not tr.any() and not tp.any()


# -- walls -------------------------------------------------------------------------
def test_wall_test_sphere_margin():
    s = _setup()
    q = np.array([1.0, 0, 0, 0])
    a = 0.01
    rc, wn, arm, dx, isect = po.wall_boundary_condition(s, a, 1.0, [0.5 * a, 1.0, 1.0], q)
    assert rc == 0 and isect == 1 and wn[0] == 1.0
    assert np.allclose(arm, [a, 0, 0]) and np.isclose(dx, 0.5 * a)
    rc, wn, arm, dx, isect = po.wall_boundary_condition(s, a, 1.0, [1.1 * a, 1.0, 1.0], q)
    assert isect == 0 and not arm.any()


def test_wall_rebound_elastic_energy():
    s = _setup(ecw=1.0, muw=0.0)
    rng = np.random.default_rng(6)
    q = _unit_q(rng)
    rc, u, om = po.wall_rebound(s, (1e-5, 2e-5, 2e-5), [-1.0, 0.2, 0.1], [3.0, -1.0, 0.5], q,
                                [0.004, 0.001, -0.002], [1.0, 0, 0])
    assert rc == 0
    assert u[0] > 0


# -- contacts ------------------------------------------------------------------------
def test_sphere_start_is_stationary():
    """ellipsoid_contact_detection.f90:77-87 starts from n = (b1-b2)/|b1-b2|, where
    the support points face away from each other.  For spheres that direction is a
    stationary point (the largest gap): the Jacobian vanishes up to rounding and lmder
    stops there, so overlapping spheres are not reported in contact; the restatement
    keeps that."""
    q = np.array([1.0, 0, 0, 0])
    r = 0.01
    for d in (0.015, 0.019):
        res = po.contact_detection(r, 1.0, r, 1.0, [0, 0, 0], q, [d, 0, 0], q)
        assert res["flag"] == 0 and res["info"] in (1, 4)
        gap = np.linalg.norm(res["ept1"] - res["ept2"])
        assert abs(gap - (2 * r + d)) < 1e-12


def test_reported_contacts_are_real_overlaps():
    """Soundness: whenever the solve reports contact, the two bodies overlap (checked
    by dense sampling of the segment between the two contact points)."""
    rng = np.random.default_rng(12)
    hits = 0
    for _ in range(300):
        a1, a2 = rng.uniform(0.005, 0.02, 2)
        p1, p2 = rng.uniform(0.3, 4, 2)
        b1 = rng.uniform(0, 1, 3)
        d = rng.normal(size=3); d /= np.linalg.norm(d)
        b2 = b1 + d * (max(a1, a1 / p1) + max(a2, a2 / p2)) * rng.uniform(0.2, 1.0)
        q1, q2 = _unit_q(rng), _unit_q(rng)
        res = po.contact_detection(a1, p1, a2, p2, b1, q1, b2, q2)
        if res["flag"]:
            hits += 1
            assert po.fmargin(a1, p1, res["ept2"], b1, q1) < 1.0
            assert po.fmargin(a2, p2, res["ept1"], b2, q2) < 1.0
            mid = 0.5 * (res["ept1"] + res["ept2"])
            assert po.fmargin(a1, p1, mid, b1, q1) < 1.0 and po.fmargin(a2, p2, mid, b2, q2) < 1.0
    assert hits > 20


def test_lm_matches_scipy_minpack_bitwise():
    """The restated solver is MINPACK's lmder: with the same residual and Jacobian,
    scipy's MINPACK returns the same iterate, info code and evaluation count."""
    from scipy.optimize import leastsq
    L = po.lib()
    L.orc_contact_lm.restype = C.c_int32
    rng = np.random.default_rng(7)
    tol = np.sqrt(np.finfo(float).eps)
    checked = 0
    while checked < 60:
        a1, a2 = rng.uniform(0.005, 0.02, 2)
        p1, p2 = rng.uniform(0.3, 4, 2)
        b1 = rng.uniform(0, 1, 3)
        d = rng.normal(size=3); d /= np.linalg.norm(d)
        b2 = b1 + d * (max(a1, a1 / p1) + max(a2, a2 / p2)) * rng.uniform(0.2, 1.1)
        q1, q2 = _unit_q(rng), _unit_q(rng)
        args = [C.c_double(a1), C.c_double(p1), C.c_double(a2), C.c_double(p2), po.dptr(b1), po.dptr(q1),
                po.dptr(b2), po.dptr(q2)]
        cn = (b1 - b2) / np.linalg.norm(b1 - b2)
        x0 = np.array([np.arccos(cn[0] / np.cos(np.arcsin(cn[2]))), np.arcsin(cn[2])])
        if np.isnan(x0).any():
            continue
        def f(x):
            x = np.ascontiguousarray(x, dtype=np.float64); o = np.zeros(3)
            L.orc_contact_residual(*args, po.dptr(x), po.dptr(o)); return o
        def j(x):
            x = np.ascontiguousarray(x, dtype=np.float64); o = np.zeros(6)
            L.orc_contact_jacobian(*args, po.dptr(x), po.dptr(o)); return o.reshape(2, 3).T.copy()
        xs, _, info, _, ier = leastsq(f, x0.copy(), Dfun=j, full_output=True, ftol=tol, xtol=tol, gtol=0.0,
                                      maxfev=300, factor=100)
        xm = x0.copy()
        nf = C.c_int32()
        got = L.orc_contact_lm(*args, po.dptr(xm), C.c_double(tol), C.byref(nf))
        assert np.array_equal(xs, xm)
        assert got == (4 if ier == 8 else ier) and nf.value == info["nfev"]
        checked += 1


def test_contact_golden_vectors():
    """Committed scipy/MINPACK solutions (numpy residual and Jacobian written
    independently of the oracle)."""
    data = json.load(open(os.path.join(HERE, "golden", "lm_contact.json")))
    L = po.lib()
    L.orc_contact_lm.restype = C.c_int32
    for c in data["cases"]:
        x = np.array(c["x0"])
        args = [C.c_double(c["emaj1"]), C.c_double(c["apr1"]), C.c_double(c["emaj2"]), C.c_double(c["apr2"]),
                po.dptr(np.array(c["b1"])), po.dptr(np.array(c["q1"])), po.dptr(np.array(c["b2"])),
                po.dptr(np.array(c["q2"]))]
        nf = C.c_int32()
        L.orc_contact_lm(*args, po.dptr(x), C.c_double(data["tol"]), C.byref(nf))
        # the fixture's residual rounds differently, so the two solves stop at points
        # that agree to the solver tolerance (xtol = sqrt(eps)), not bitwise
        assert np.allclose(x, c["x"], rtol=0, atol=20 * data["tol"]), (x, c["x"])
        res = po.contact_detection(c["emaj1"], c["apr1"], c["emaj2"], c["apr2"], c["b1"], c["q1"], c["b2"], c["q2"])
        if abs(c["contact"]) > 1e-9:
            assert (res["flag"] == 1) <= (c["contact"] > 0)   # contact requires positive depth


def test_collision_response_conserves_momentum_and_energy():
    s = _setup(ecp=1.0, mup=0.0)
    rng = np.random.default_rng(8)
    ip = (2e-6, 5e-6, 5e-6)
    for _ in range(20):
        q1, q2 = _unit_q(rng), _unit_q(rng)
        u1, u2 = rng.normal(size=3), rng.normal(size=3)
        o1, o2 = rng.normal(size=3) * 10, rng.normal(size=3) * 10
        n = rng.normal(size=3); n /= np.linalg.norm(n)
        r1, r2 = rng.normal(size=3) * 0.003, rng.normal(size=3) * 0.003
        rc, a1, b1, a2, b2 = po.collision_response(s, ip, u1, o1, q1, u2, o2, q2, r1, r2, n)
        assert rc == 0
        assert np.allclose(a1 + a2, u1 + u2, atol=1e-12)   # equal unit masses


# -- collision grid ------------------------------------------------------------------
def _grid_ensemble(n_boxes_edge=6, n=200, seed=9):
    L = 2 * np.pi
    s = config.Setup(nx=16, ny=16, nz=16, lx=L, ly=L, lz=L)
    rng = np.random.default_rng(seed)
    emaj = np.full(n, L / n_boxes_edge / 4.0 * 0.999)
    st = {"x": rng.random(n) * L, "y": rng.random(n) * L, "z": rng.random(n) * L,
          "emaj": emaj, "apr": np.full(n, 2.0), "rhop": np.full(n, 1000.0),
          "ipxx": np.ones(n), "ipyy": np.ones(n), "ipzz": np.ones(n)}
    for k in ("u", "v", "w", "ox", "oy", "oz", "qb", "qc", "qd"):
        st[k] = np.zeros(n)
    st["qa"] = np.ones(n)
    return po.Ensemble(s, st)


def test_half_stencil_visits_each_adjacent_box_pair_once():
    ens = _grid_ensemble()
    g = ens.boxgrid()
    ncon, con = ens.connectivity(g)
    assert (ncon == 13).all()
    nx, ny, nz = g.nxbox, g.nybox, g.nzbox
    seen = {}
    for b in range(g.nbox):
        for v in con[b * 27:b * 27 + ncon[b]]:
            key = tuple(sorted((b, v - 1)))
            seen[key] = seen.get(key, 0) + 1
    assert all(c == 1 for c in seen.values())
    def coords(b):
        return b % nx, (b // nx) % ny, b // (nx * ny)
    for (a, b) in list(seen)[:500]:
        ca, cb = coords(a), coords(b)
        for d, m in zip((cb[0] - ca[0], cb[1] - ca[1], cb[2] - ca[2]), (nx, ny, nz)):
            assert d % m in (0, 1, m - 1)
    assert len(seen) == 13 * g.nbox


def test_detected_pairs_match_brute_force_box_rule():
    ens = _grid_ensemble(n=400)
    g = ens.boxgrid()
    home, near = po.detect_pairs(ens)
    rc, ijk = po.box_index(ens, g)
    assert rc == 0
    nx, ny, nz = g.nxbox, g.nybox, g.nzbox
    b = ijk - 1
    bc = np.stack([b % nx, (b // nx) % ny, b // (nx * ny)], 1)
    brute = set()
    for i, j in itertools.combinations(range(ens.n), 2):
        d = (bc[j] - bc[i] + [nx, ny, nz]) % [nx, ny, nz]
        if all(x in (0, 1, m - 1) for x, m in zip(d, (nx, ny, nz))):
            brute.add((i, j))
    got = {tuple(sorted(p)) for p in zip(home.tolist(), near.tolist())}
    assert got == brute
    assert len(home) == len(brute)


def test_serial_and_parallel_collision_agree():
    s = config.Setup(nx=32, ny=32, nz=32, visc=0.05)
    spec = config.ParticleSpec(n=3000, ar_range=(0.5, 3.0), b=0.05, st=1.0, seed=3)
    st = particles.draw(spec, s)
    a = po.Ensemble(s, st)
    b = po.Ensemble(s, st)
    ra = a.collide(prefilter=True, nthreads=1)
    rb = b.collide(prefilter=False, nthreads=4)
    assert ra["n_coll"] > 0
    assert np.array_equal(ra["home"], rb["home"]) and np.array_equal(ra["near"], rb["near"])
    for k in po.STATE_KEYS:
        assert np.array_equal(a.a[k], b.a[k])


# -- statistics beside the step ------------------------------------------------
# a generic line of centres: the contact solve's initial guess degenerates when the
# centre line lies along x (it converges to the opposite normal) or has no y part
# (acos of an undefined ratio), as the reference's does (Q14)
_E = np.array([0.6, 0.48, 0.64])


def _spheres(ss, us, a=0.05):
    """Spheres centred at 3 + s e with velocity u e, for s in ss and u in us."""
    n = len(ss)
    s = config.Setup(nx=32, ny=32, nz=32, visc=0.05, dtime=1e-3)
    st = {k: np.zeros(n) for k in po.STATE_KEYS}
    for j, k in enumerate(("x", "y", "z")):
        st[k] = 3.0 + np.array(ss, dtype=float) * _E[j]
    for j, k in enumerate(("u", "v", "w")):
        st[k] = np.array(us, dtype=float) * _E[j]
    st["qa"][:] = 1.0
    st["emaj"] = np.full(n, a)
    st["apr"] = np.ones(n)
    st["rhop"] = np.full(n, 1000.0)
    for k in ("ipxx", "ipyy", "ipzz"):
        st[k] = np.full(n, 2.0 * a * a / 5.0)
    return s, st


def test_collision_stats_head_on_spheres():
    """Two overlapping spheres closing head on: one contact, one collision, depth
    2a - d, NVREL = -|v_rel|, angle pi (collision_interaction.f90:330-345), to the
    accuracy of the contact solve (its residual is the squared depth, so the normal
    settles within about 1e-2 rad of the centre line)."""
    a, d, v = 0.05, 0.09, 0.3
    s, st = _spheres([3.0, 3.0 + d], [v, -v], a)
    rc, cs, ncoll = po.Ensemble(s, st).collide_stats()
    assert rc == 0 and ncoll == 1
    c = cs[0, 0]
    assert c[0] == 1.0 and c[1] == 1.0 and c[2] == 2.0 / s.dtime
    assert abs(c[3] - (2 * a - d)) < 1e-2 * (2 * a - d) and c[4] == c[3]
    assert abs(c[5] + 2 * v) < 1e-3 * v and abs(c[6] - 2 * v) < 1e-12
    assert abs(c[7] - np.pi) < 2e-2


def test_collision_stats_count_only_examined_pairs():
    """Three spheres in a row, both contacts closing: the COLOR walk accepts the first
    pair and never examines the second, so one contact is counted although the two
    pairs are in contact; the indices split the sums by (IDP of HOME, IDP of NEAR)."""
    a, d, v = 0.05, 0.09, 0.3
    s, st = _spheres([3.0, 3.0 + d, 3.0 + 2 * d], [v, 0.0, -v], a)
    ens = po.Ensemble(s, st)
    full = po.Ensemble(s, st).collide(prefilter=True, nthreads=1)
    assert full["n_contacts"] == 1 and full["n_coll"] == 1        # the walk evaluates one pair
    every = po.Ensemble(s, st).collide(prefilter=True, nthreads=4)
    assert every["n_contacts"] == 2                                # both pairs are in contact
    rc, cs, ncoll = ens.collide_stats(group=np.array([1, 2, 2]), ngroups=2)
    assert rc == 0 and ncoll == 1
    assert cs[:, :, 0].sum() == 1.0 and cs[:, :, 1].sum() == 1.0
    h, nr = full["home"][0], full["near"][0]
    g = np.array([1, 2, 2]) - 1
    assert cs[g[h], g[nr], 0] == 1.0


def test_stat_partfluid_known_values():
    """A sphere at rest in a uniform stream U along x: Re_p = U d / visc, no lift, drag
    along x, phi = 0, symmetry axis x; tau_p of a sphere (FBETA = 1)."""
    s = config.Setup(nx=32, ny=32, nz=32, visc=0.05)
    a, rhop, U = 0.01, 1000.0, 0.7
    v = np.zeros(36)
    po.lib().orc_stat_partfluid_particle(C.byref(po.make_setup(s)), C.c_double(a), C.c_double(1.0),
                                         C.c_double(rhop), po.dptr(np.zeros(3)), po.dptr(np.zeros(3)),
                                         po.dptr(np.array([1.0, 0, 0, 0])), po.dptr(np.array([U, 0, 0])),
                                         po.dptr(np.zeros(3)), po.dptr(v))
    d = 2 * a
    assert abs(v[0] - U * d / s.visc) < 1e-12 * v[0]
    assert v[24] == 0.0 and v[25] == 1.0 and v[26] == 0.0 and v[27] == 0.0
    assert v[3] > 0 and v[4] == 0.0 and v[5] == 0.0                  # drag along the stream
    assert v[6] == 0.0 or np.isnan(v[7])                           # no transverse lift (0/0 there)
    assert abs(v[22] - (2.0 / 9.0) * rhop * a * a / (s.rhof * s.visc)) < 1e-12 * v[22]
    assert v[35] == 1.0 and v[29] == 0.0


def test_solve_lengths_persist_between_steps():
    """The contact queue's premise, on the oracle: at the 512^3 workload's particle density
    and sizes (a periodic sample of 4,096 spheroids), nearly every pair whose bounding
    spheres overlap in a step overlapped in the step before, and the Levenberg-Marquardt
    evaluation counts of the same pair in two consecutive steps correlate strongly."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    w = config.WORKLOADS["c3_512cube_n16777216_fp32field"]
    ens, refs, g = bench.cpu_sample(w, 16, bench.workload_max_emaj(w))
    L = ens.setup.lx

    def solve_lengths():
        a = ens.a
        home, near = po.detect_pairs(ens)
        d = np.stack([a[k][near] - a[k][home] for k in ("x", "y", "z")], 1)
        d -= L * np.round(d / L)
        rb = lambda i: np.maximum(a["emaj"][i], a["emaj"][i] / a["apr"][i])   # noqa: E731
        ok = (d * d).sum(1) <= (rb(home) + rb(near)) ** 2
        out = {}
        for e in np.flatnonzero(ok):
            i1, i2 = int(home[e]), int(near[e])
            b1 = np.array([a["x"][i1], a["y"][i1], a["z"][i1]])
            q = [np.array([a[k][i] for k in ("qa", "qb", "qc", "qd")]) for i in (i1, i2)]
            r = po.contact_detection(a["emaj"][i1], a["apr"][i1], a["emaj"][i2], a["apr"][i2],
                                     b1, q[0], b1 + d[e], q[1])
            out[(i1, i2)] = r["nfev"]
        return out

    first = solve_lengths()
    assert ens.advance(refs, nthreads=4) == 0
    assert ens.collide(prefilter=True, nthreads=4, grid=g)["rc"] == 0
    second = solve_lengths()
    both = [k for k in second if k in first]
    assert len(second) >= 50
    assert len(both) >= 0.9 * len(second)
    a = np.array([first[k] for k in both], dtype=float)
    b = np.array([second[k] for k in both], dtype=float)
    assert np.corrcoef(a, b)[0, 1] > 0.6
