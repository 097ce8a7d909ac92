"""The per-routine drop-ins of the C ABI against the oracle, on thousands of seeded
inputs each, edge cases included, through the same entry points a Fortran wrapper binds.

| entry point | reference | bar |
|---|---|---|
| gp_fluid_force_ellipsoid[_batch] | fluid_force_ellipsoid.f90:1-161 | 1e-12 relative (libm pow/atan/sin/cos) |
| gp_fluid_torque_ellipsoid[_batch] | fluid_torque_ellipsoid.f90:1-190 | 1e-12 relative |
| gp_quaternion_integration[_batch] | adv_quaternion.f90:1-117 | 1e-12 relative |
| gp_euler_integration | adv_angular_velocity.f90:113-144 | bit for bit |
| gp_collision_box_connectivity | collision_box_connectivity.f90:7-384 | bit for bit |
| gp_ellipsoid_contact_detection[_batch] | ellipsoid_contact_detection.f90:1-187 | bit for bit |
| gp_collision_response | collision_response.f90:1-437 | bit for bit |

The force, torque and quaternion routines call pow, atan, sin and cos; the device's math
library and the host's may differ by an ulp there, so those are held to the state
tolerance.  The others use only IEEE-rounded operations (and the contact solve's own
trigonometry, shared with the oracle) and must agree exactly."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle as po
from gazpart_b200 import api, config

pytestmark = pytest.mark.gpu

TOL = 1e-12
# (IG, IDP) -> EMAJ, APR, RHOP: oblate, sphere, prolate, slender
CLASSES = {(1, 1): (0.01, 0.25, 800.0), (1, 2): (0.02, 1.0, 1000.0), (2, 1): (0.015, 3.0, 1200.0),
           (2, 2): (0.03, 5.0, 2500.0)}


def _ctx(setup=None):
    setup = setup or config.Setup(nx=32, ny=32, nz=32, visc=0.0184, dtime=1e-3)
    ctx = api.Context(setup, "fp64")
    for (ig, idp), (emaj, apr, rhop) in CLASSES.items():
        ctx.set_class(ig, idp, emaj, apr, rhop)
    return setup, ctx


def _unit_quats(rng, n):
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def _classes(rng, n):
    keys = list(CLASSES)
    pick = rng.integers(0, len(keys), n)
    ig = np.array([keys[k][0] for k in pick], dtype=np.int32)
    idp = np.array([keys[k][1] for k in pick], dtype=np.int32)
    return ig, idp, [CLASSES[keys[k]] for k in pick]


def _vec_rel(a, b):
    """max over rows of |a - b| / |b| (rows of 3), NaN equal to NaN."""
    both_nan = np.isnan(a) & np.isnan(b)
    assert np.array_equal(np.isnan(a), np.isnan(b))
    d = np.where(both_nan, 0.0, a - b)
    nb = np.linalg.norm(np.where(both_nan, 0.0, b), axis=1)
    nd = np.linalg.norm(d, axis=1)
    scale = np.maximum(nb, 1e-300)
    return float(np.max(np.where(nd == 0.0, 0.0, nd / scale)))


def _same(a, b):
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


def _force_inputs(rng, n):
    up = rng.normal(size=(n, 3))
    uf = rng.normal(size=(n, 3))
    q = _unit_quats(rng, n)
    # Q7 edges: zero relative velocity (guard: no force), and a relative velocity along
    # the symmetry axis (no transverse part: no lift), and a tiny relative velocity
    up[:20] = uf[:20]
    axis = np.stack([1 - 2 * (q[:, 2] ** 2 + q[:, 3] ** 2), 2 * (q[:, 1] * q[:, 2] + q[:, 0] * q[:, 3]),
                     2 * (q[:, 1] * q[:, 3] - q[:, 0] * q[:, 2])], 1)
    up[20:40] = uf[20:40] + 0.3 * axis[20:40]
    up[40:60] = uf[40:60] + 1e-9 * rng.normal(size=(20, 3))
    return up, uf, q


def test_fluid_force_ellipsoid():
    rng = np.random.default_rng(101)
    n = 4000
    up, uf, q = _force_inputs(rng, n)
    setup, ctx = _ctx()
    with ctx:
        ig, idp, props = _classes(rng, n)
        fd, fl = ctx.fluid_force_ellipsoid(ig, idp, up, uf, q)
        rd, rl = np.empty((n, 3)), np.empty((n, 3))
        for i in range(n):
            rc, rd[i], rl[i] = po.fluid_force(setup, *props[i], up[i], uf[i], q[i])
            assert rc == 0
        # the reference's argument list (IG, IDP, UPART..WFLUID, quat) for single particles
        L = api._lib.lib()
        for i in (0, 25, 45, 3999):
            d, l = np.empty(3), np.empty(3)
            qi = np.ascontiguousarray(q[i])
            rc = L.gp_fluid_force_ellipsoid(ctx._h, int(ig[i]), int(idp[i]), *[float(v) for v in up[i]],
                                            *[float(v) for v in uf[i]], qi.ctypes.data_as(api._lib._dp),
                                            d.ctypes.data_as(api._lib._dp), l.ctypes.data_as(api._lib._dp))
            assert rc == 0
            assert np.array_equal(d, fd[i]) and np.array_equal(l, fl[i])
        ctx.raise_status()
    assert np.all(fd[:20] == 0.0) and np.all(fl[:20] == 0.0)      # zero slip: no force
    assert np.all(np.abs(fl[20:40]) < 1e-12 * (1 + np.abs(fd[20:40])))   # axial slip: no lift
    assert _vec_rel(fd, rd) < TOL and _vec_rel(fl, rl) < TOL, (_vec_rel(fd, rd), _vec_rel(fl, rl))


def test_fluid_torque_ellipsoid():
    rng = np.random.default_rng(102)
    n = 4000
    up, uf, q = _force_inputs(rng, n)
    vort = rng.normal(size=(n, 3)) * 3.0
    om = rng.normal(size=(n, 3)) * 2.0
    om[60:80] = 0.0                        # Q7: no relative spin (zero rotational Reynolds number)
    vort[60:80] = 0.0
    setup, ctx = _ctx()
    with ctx:
        ig, idp, props = _classes(rng, n)
        tp, tr = ctx.fluid_torque_ellipsoid(ig, idp, om, q, up, uf, vort)
        ctx.raise_status()
    rp, rr = np.empty((n, 3)), np.empty((n, 3))
    for i in range(n):
        rc, rp[i], rr[i] = po.fluid_torque(setup, *props[i], up[i], uf[i], vort[i], om[i], q[i])
        assert rc == 0
    assert _vec_rel(tp, rp) < TOL and _vec_rel(tr, rr) < TOL, (_vec_rel(tp, rp), _vec_rel(tr, rr))


def test_quaternion_integration():
    rng = np.random.default_rng(103)
    n = 5000
    q = _unit_quats(rng, n)
    q[:50] *= 1.1                             # Q15: a non-unit quaternion keeps its norm
    om = rng.normal(size=(n, 3)) * 20.0
    om[50:70] = 0.0                           # no rotation
    om[70:90] *= 1e-12
    dt = 5e-4
    setup, ctx = _ctx()
    with ctx:
        got = ctx.quaternion_integration(q, om, dt)
    ref = np.array([po.quaternion_integration(q[i], om[i], dt) for i in range(n)])
    assert np.array_equal(got[50:70], q[50:70])
    d = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert float(d.max()) < TOL, float(d.max())


def test_euler_integration_bit_exact():
    """EULER_INTEGRATION (the dry path; RK4 on the torque-free Euler equations) uses only
    IEEE arithmetic, so the device and the oracle agree exactly."""
    rng = np.random.default_rng(104)
    setup, ctx = _ctx()
    with ctx:
        for (ig, idp), (emaj, apr, rhop) in CLASSES.items():
            a = emaj
            b = a / apr
            ip = ((b * b + b * b) / 5.0, (a * a + b * b) / 5.0, (a * a + b * b) / 5.0)
            for _ in range(50):
                om = rng.normal(size=3) * 10.0
                got = ctx.euler_integration(ig, idp, om)
                ref = po.euler_integration(ip, om, setup.dtime)
                assert np.array_equal(got, ref), (ig, idp, got, ref)


def _box_case(lx, ly, lz, nbox, periodic):
    """A context whose box grid has about nbox boxes along x: COLLISION_INITIATION sizes
    boxes from DPMAX = 2 EMAJ_max (collision_initiation.f90:50-78)."""
    emaj = lx / (4.0 * nbox + 2.0)
    setup = config.Setup(nx=16, ny=16, nz=16, lx=lx, ly=ly, lz=lz, periodicity=periodic)
    st = {k: np.zeros(4) for k in api.STATE_KEYS}
    st["qa"][:] = 1.0
    st["x"][:] = [0.1 * lx, 0.3 * lx, 0.5 * lx, 0.7 * lx]
    st["y"][:] = 0.5 * ly
    st["z"][:] = 0.5 * lz
    for k, v in (("emaj", emaj), ("apr", 2.0), ("rhop", 1000.0)):
        st[k] = np.full(4, v)
    a, b = emaj, emaj / 2.0
    st["ipxx"] = np.full(4, (b * b + b * b) / 5.0)
    st["ipyy"] = np.full(4, (a * a + b * b) / 5.0)
    st["ipzz"] = np.full(4, (a * a + b * b) / 5.0)
    return setup, st


@pytest.mark.parametrize("lx,ly,lz,nbox,periodic", [
    (2 * np.pi, 2 * np.pi, 2 * np.pi, 3, True), (2 * np.pi, 2 * np.pi, 2 * np.pi, 4, True),
    (2 * np.pi, 2 * np.pi, 2 * np.pi, 9, True), (2 * np.pi, 2 * np.pi, 2 * np.pi, 3, False),
    (2 * np.pi, 2 * np.pi, 2 * np.pi, 5, False), (2 * np.pi, np.pi, 3 * np.pi, 7, True),
    (2 * np.pi, np.pi, 3 * np.pi, 6, False), (1.0, 2.0, 0.5, 17, True)])
def test_collision_box_connectivity_bit_exact(lx, ly, lz, nbox, periodic):
    setup, st = _box_case(lx, ly, lz, nbox, periodic)
    with api.Context(setup, "fp64") as ctx:
        ctx.upload(st)
        got = ctx.collision_box_connectivity()
    ens = po.Ensemble(setup, st)
    g = ens.boxgrid()
    ncon, con = ens.connectivity(g)
    assert list(got["dims"]) == [g.nxbox, g.nybox, g.nzbox]
    assert got["geom"].tolist() == [g.dxbox, g.dybox, g.dzbox, g.xminbox, g.yminbox, g.zminbox]
    assert np.array_equal(got["ncon"], ncon)
    assert np.array_equal(got["con"], con)
    assert g.nxbox == nbox


def test_collision_box_grid_below_three_boxes_is_refused():
    """With fewer than three boxes along a direction the half stencil would list one
    neighbour twice (collision_box_connectivity.f90:59-73 wraps both ways onto the same
    box); the library refuses such a grid instead of producing duplicate pairs."""
    setup, st = _box_case(2 * np.pi, 2 * np.pi, 2 * np.pi, 2, True)
    with api.Context(setup, "fp64") as ctx:
        with pytest.raises(api.GPError):
            ctx.upload(st)


def _contact_pairs(rng, n):
    shapes = np.empty((n, 4))
    keys = list(CLASSES)
    for i in range(n):
        e1, a1, _ = CLASSES[keys[rng.integers(0, len(keys))]]
        e2, a2, _ = CLASSES[keys[rng.integers(0, len(keys))]]
        shapes[i] = (e1, a1, e2, a2)
    q = np.hstack([_unit_quats(rng, n), _unit_quats(rng, n)])
    b1 = rng.uniform(0.0, 1.0, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    reach = (np.maximum(shapes[:, 0], shapes[:, 0] / shapes[:, 1])
             + np.maximum(shapes[:, 2], shapes[:, 2] / shapes[:, 3]))
    b2 = b1 + d * (reach * rng.uniform(0.1, 1.1, n))[:, None]
    # Q14: centre lines in the x-z plane, where the starting angle can be NaN
    for i in range(40):
        t = 0.05 + 1.4 * i / 40.0
        nrm = np.array([np.cos(t), 0.0, np.sin(t)])
        shapes[i] = (0.05, 1.5, 0.05, 1.5)
        q[i, :4] = (1.0, 0.0, 0.0, 0.0)
        q[i, 4:] = np.array([0.9, 0.3, 0.2, 0.1]) / np.linalg.norm([0.9, 0.3, 0.2, 0.1])
        b1[i] = 0.0
        b2[i] = -0.05 * nrm
    return shapes, np.hstack([b1, b2]), q


def test_ellipsoid_contact_detection_bit_exact():
    rng = np.random.default_rng(105)
    n = 3000
    shapes, centres, quats = _contact_pairs(rng, n)
    setup, ctx = _ctx()
    with ctx:
        flag, e1, e2, cn = ctx.ellipsoid_contact_detection(shapes, centres, quats)
        # the reference's argument list (IG, IDP1, IDP2, centres, quaternions) for a few pairs
        one = {}
        for i in (100, 200, 300):
            f = (api.C.c_int32(), np.empty(3), np.empty(3), np.empty(3))
            ig, idp1, idp2 = 2, 1, 2
            sh = (CLASSES[(2, 1)][0], CLASSES[(2, 1)][1], CLASSES[(2, 2)][0], CLASSES[(2, 2)][1])
            c = centres[i]
            qq = quats[i]
            rc = api._lib.lib().gp_ellipsoid_contact_detection(
                ctx._h, ig, idp1, idp2, c[0], c[1], c[2], qq[:4].ctypes.data_as(api._lib._dp), c[3], c[4], c[5],
                np.ascontiguousarray(qq[4:]).ctypes.data_as(api._lib._dp), api.C.byref(f[0]),
                f[1].ctypes.data_as(api._lib._dp), f[2].ctypes.data_as(api._lib._dp),
                f[3].ctypes.data_as(api._lib._dp))
            assert rc == 0
            one[i] = (f[0].value, f[1], f[2], f[3], po.contact_detection(*sh, c[:3], qq[:4], c[3:], qq[4:]))
    nan_start = 0
    for i in range(n):
        s, c, q = shapes[i], centres[i], quats[i]
        r = po.contact_detection(s[0], s[1], s[2], s[3], c[:3], q[:4], c[3:], q[4:])
        assert flag[i] == r["flag"], i
        assert _same(e1[i], r["ept1"]) and _same(e2[i], r["ept2"]) and _same(cn[i], r["cnormal"]), i
        nan_start += int(np.isnan(r["x"][0]))
    assert 0 < int(flag.sum()) < n
    assert nan_start > 0                      # the Q14 start was met
    for i, (fl, a, b, nn, r) in one.items():
        assert fl == r["flag"] and _same(a, r["ept1"]) and _same(b, r["ept2"]) and _same(nn, r["cnormal"]), i


@pytest.mark.parametrize("ecp,mup", [(1.0, 0.0), (0.9, 0.3)])
def test_collision_response_bit_exact(ecp, mup):
    """COLLISION_RESPONSE with the inertia of class (IG, IDP) for both bodies (Q8).  With
    e < 1 or friction the reference's energy balance stops the run (Q9): both sides report
    it (GP_EENERGY) and still agree on the updated velocities."""
    rng = np.random.default_rng(106 + int(10 * ecp))
    setup = config.Setup(nx=32, ny=32, nz=32, ecp=ecp, mup=mup)
    setup, ctx = _ctx(setup)
    rcs = set()
    with ctx:
        for t in range(400):
            (ig, idp) = list(CLASSES)[t % len(CLASSES)]
            emaj, apr, _ = CLASSES[(ig, idp)]
            a, b = emaj, emaj / apr
            ip = ((b * b + b * b) / 5.0, (a * a + b * b) / 5.0, (a * a + b * b) / 5.0)
            u1, o1, u2, o2 = (rng.normal(size=3) for _ in range(4))
            q1, q2 = _unit_quats(rng, 2)
            nrm = rng.normal(size=3)
            nrm /= np.linalg.norm(nrm)
            r1 = -nrm * emaj * rng.uniform(0.3, 1.0) + rng.normal(size=3) * 0.1 * emaj
            r2 = nrm * emaj * rng.uniform(0.3, 1.0) + rng.normal(size=3) * 0.1 * emaj
            p1 = np.concatenate([u1, o1, q1])
            p2 = np.concatenate([u2, o2, q2])
            rc, g1, g2 = ctx.collision_response(ig, idp, p1, p2, r1, r2, nrm)
            rrc, ru1, ro1, ru2, ro2 = po.collision_response(setup, ip, u1, o1, q1, u2, o2, q2, r1, r2, nrm)
            assert rc == rrc, t
            rcs.add(rc)
            assert np.array_equal(g1[:3], ru1) and np.array_equal(g1[3:6], ro1), t
            assert np.array_equal(g2[:3], ru2) and np.array_equal(g2[3:6], ro2), t
            assert np.array_equal(g1[6:], q1) and np.array_equal(g2[6:], q2)
    if ecp == 1.0 and mup == 0.0:
        assert rcs == {0}
    else:
        assert 3 in rcs                       # GP_EENERGY: the reference's energy stop
