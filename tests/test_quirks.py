"""Reference quirks that the oracle reproduces, one test each where the quirk can be
isolated on the CPU.  The GPU parity tests hold the device path to the oracle bit for
bit, so these behaviours carry over to it.

Quirks covered elsewhere:
- Q5 (DX = L/(N-1), index period N): test_oracle.test_interp_at_nodes_is_exact.
- Q6 (vorticity ghosts read zero): test_host.test_reference_layout_ghosts.
- Q7 (zero relative speed): test_oracle.test_force_guard_and_drag_direction.
- Q13 (greedy COLOR order): test_oracle.test_serial_and_parallel_collision_agree.
- Q16 (param.in against the reader): test_files.
- Q18 (mirror boundary): test_oracle.test_frozen_interp_mirror_matches_interior."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

import pyoracle as po
from gazpart_b200 import config, field

L = 2.0 * np.pi


def _quiet_field(s):
    """Reference-layout arrays of a fluid at rest, for single-particle steps."""
    z = torch.zeros(s.nz, s.ny, s.nx, dtype=torch.float64)
    return [field.reference_layout(z, "periodic" if c < 3 else "zero").numpy().copy() for c in range(6)]


def _one(s, emaj, apr, x, u, om, q=(1.0, 0.0, 0.0, 0.0)):
    """A one-particle ensemble with the reference's per-particle constants."""
    from gazpart_b200 import particles
    st = particles.draw(config.ParticleSpec(n=1, ar=apr, b=emaj / apr, st=1.0, seed=3), s)
    st["x"][0], st["y"][0], st["z"][0] = x
    st["u"][0], st["v"][0], st["w"][0] = u
    st["ox"][0], st["oy"][0], st["oz"][0] = om
    st["qa"][0], st["qb"][0], st["qc"][0], st["qd"][0] = q
    return po.Ensemble(s, st)


def test_q1_wall_test_runs_in_a_periodic_box():
    """Q1 (adv_particle_new.f90:331-336,555-560): the x = 0 and x = L planes are tested
    even with PERIODICITY, so a particle closing on x = 0 rebounds instead of wrapping."""
    s = config.Setup(nx=16, ny=16, nz=16, visc=0.05, dtime=1e-3, periodicity=True)
    ens = _one(s, 0.05, 1.5, (0.0504, 3.0, 3.0), (-0.8, 0.0, 0.0), (0.0, 0.0, 0.0))
    # the symmetry axis lies along x (q = 1), so the x extent is the major semi-axis and
    # the predictor position crosses x = 0
    assert 0.0504 - 1e-3 * 0.8 < ens.a["emaj"][0]
    assert ens.advance(_quiet_field(s)) == 0
    assert ens.a["u"][0] > 0.0                             # rebounded
    assert 0.0 < ens.a["x"][0] < 1.0                       # not wrapped to x near L


def test_q1_rebound_of_a_slender_spheroid_stops_the_run_at_dt_5e4():
    """Q1 with the 512^3 / 16.8M workload's viscosity and time step (dt = 5e-4): a slender
    spheroid of that workload's distribution (AR 4.65, EMAJ 4.1e-3) closing on x = 0 in
    the periodic box rebounds off the plane (adv_particle_new.f90:331-336), which spins it
    to about 1.7e3 rad/s.  The explicit RK2 update of its angular velocity
    (adv_particle_new.f90:278-320,516-632) is then unstable at this time step: |omega|
    grows about twofold per step until the drag is NaN and the reference stops with 'In
    Fluid force' (fluid_force_ellipsoid.f90:150-159), 25 steps in.  The same particle in
    the middle of the box runs on.  This is why the benchmark starts its particles away
    from the x planes (the x margin of its configuration)."""
    w = config.C3
    base = w.setup()
    s = config.Setup(nx=64, ny=64, nz=64, visc=base.visc, dtime=base.dtime)
    assert s.dtime == 5e-4
    f = field.generate(64, seed=0, device="cpu")
    refs = [field.reference_layout(f[k], "periodic" if k in ("u", "v", "w") else "zero").numpy().copy()
            for k in field.COMPONENTS_6]
    one = {"x": 6.549342494148082e-06, "y": 1.4964149544965306, "z": 2.1935648850209564,
           "u": -3.0960604761170893, "v": 1.2298512984753176, "w": -0.921259617618018,
           "qa": -0.9623316742411799, "qb": 0.0795140439437744, "qc": -0.16238840459726478,
           "qd": -0.20304007392687276, "ox": -3.2352054866547233, "oy": 3.9569619383875083,
           "oz": -4.520435237028644, "emaj": 0.004110331918409437, "apr": 4.651382660313813,
           "rhop": 3309.8084025581375, "ipxx": 3.123558465370345e-07, "ipyy": 3.535143619167598e-06,
           "ipzz": 3.535143619167598e-06}
    ens = po.Ensemble(s, {k: np.array([v]) for k, v in one.items()})
    spins = []
    rc = 0
    for step in range(40):
        rc = ens.advance(refs)
        if rc:
            break
        spins.append(float(np.sqrt(ens.a["ox"][0] ** 2 + ens.a["oy"][0] ** 2 + ens.a["oz"][0] ** 2)))
    assert rc == 1 and step == 25                          # GP_ENAN_FORCE: 'In Fluid force'
    assert 1e3 < spins[0] < 3e3                            # the rebound's spin
    growth = [spins[k + 1] / spins[k] for k in range(4, 14)]
    assert min(growth) > 1.3                               # the RK2 spin update diverges
    mid = {k: np.array([v]) for k, v in one.items()}
    mid["x"] = np.array([s.lx / 2.0])
    e2 = po.Ensemble(s, mid)
    assert all(e2.advance(refs) == 0 for _ in range(60))


def _angle(q0, q1):
    d = abs(float(np.dot(q0, q1)) / (np.linalg.norm(q0) * np.linalg.norm(q1)))
    return 2.0 * np.arccos(min(d, 1.0))


def test_q2_quaternion_advanced_twice_per_step():
    """Q2 (adv_particle_new.f90:323-325,580-582,630-632): without a rebound the step
    updates q with omega_1 after the predictor and again with omega_{n+1} from the
    predicted q, so one step turns a spinning sphere by about 2 |omega| dt."""
    s = config.Setup(nx=16, ny=16, nz=16, visc=0.05, dtime=1e-4)
    om = np.array([0.0, 0.0, 40.0])
    ens = _one(s, 0.05, 1.0, (3.0, 3.0, 3.0), (1e-3, 0.0, 0.0), om)
    q0 = np.array([ens.a[k][0] for k in ("qa", "qb", "qc", "qd")])
    assert ens.advance(_quiet_field(s)) == 0
    q1 = np.array([ens.a[k][0] for k in ("qa", "qb", "qc", "qd")])
    ratio = _angle(q0, q1) / (np.linalg.norm(om) * s.dtime)
    assert abs(ratio - 2.0) < 0.01, ratio


def _uniform_field(s, c):
    """Reference-layout arrays of a uniform flow c, with zero vorticity."""
    out = []
    for k in range(6):
        z = torch.full((s.nz, s.ny, s.nx), float(c[k]) if k < 3 else 0.0, dtype=torch.float64)
        out.append(field.reference_layout(z, "periodic" if k < 3 else "zero").numpy().copy())
    return out


def test_q3_second_stage_torque_uses_the_old_velocity():
    """Q3 (fluid_torque_ellipsoid.f90:88-105): in the corrector the force sees the
    predicted velocity u_1, but the torque reads the particle's velocity from PART, the
    step's u_n.  Rebuilding the spin update from the force and torque routines matches
    the step with u_n in the second torque and not with u_1."""
    s = config.Setup(nx=16, ny=16, nz=16, visc=0.05, dtime=5e-3)
    un = np.array([0.2, -0.1, 0.05])
    om = np.array([3.0, -2.0, 5.0])
    q0 = np.array([0.9, 0.3, 0.2, 0.1])
    q0 /= np.linalg.norm(q0)
    ens = _one(s, 0.05, 2.5, (3.0, 3.0, 3.0), un, om, q=tuple(q0))
    p = {k: ens.a[k][0] for k in ("emaj", "apr", "rhop", "ipxx", "ipyy", "ipzz")}
    assert ens.advance(_uniform_field(s, (0.7, 0.4, -0.3))) == 0
    uf = np.array([ens.a[k][0] for k in ("ufap", "vfap", "wfap")])
    vort = np.zeros(3)
    got = np.array([ens.a[k][0] for k in ("ox", "oy", "oz")])

    def k_omega(t, o):
        return np.array([(t[0] + o[1] * o[2] * (p["ipyy"] - p["ipzz"])) / p["ipxx"],
                         (t[1] + o[2] * o[0] * (p["ipzz"] - p["ipxx"])) / p["ipyy"],
                         (t[2] + o[0] * o[1] * (p["ipxx"] - p["ipyy"])) / p["ipzz"]])

    def torque(u, o, q):
        rc, tp, tr = po.fluid_torque(s, p["emaj"], p["apr"], p["rhop"], u, uf, vort, o, q)
        assert rc == 0
        return tp + tr

    rc, fd, fl = po.fluid_force(s, p["emaj"], p["apr"], p["rhop"], un, uf, q0)
    assert rc == 0
    u1 = un + s.dtime * (fd + fl)
    k1 = k_omega(torque(un, om, q0), om)
    o1 = om + s.dtime * k1
    q1 = po.quaternion_integration(q0, o1, s.dtime)
    with_un = om + 0.5 * s.dtime * (k1 + k_omega(torque(un, o1, q1), o1))
    with_u1 = om + 0.5 * s.dtime * (k1 + k_omega(torque(u1, o1, q1), o1))
    scale = np.linalg.norm(om)
    assert np.max(np.abs(got - with_un)) < 1e-13 * scale
    assert np.max(np.abs(got - with_u1)) > 1e-10 * scale


def test_q4_no_reinterpolation_at_the_predictor():
    """Q4 (adv_particle_new.f90:68-72,139-228): the field is sampled once, at x_n, and
    the corrector reuses it.  A particle whose predicted position crosses into the next
    cell would read the x plane I0+3 if the field were sampled again there; changing
    only that plane leaves the step bit for bit unchanged, while a particle already in
    that cell sees the change."""
    s = config.Setup(nx=16, ny=16, nz=16, visc=0.05, dtime=1e-3)
    m = 7
    x_below = m * s.dx - 1e-4                       # I0 = m; predictor at m*DX + 4e-4
    base = _uniform_field(s, (0.3, 0.1, -0.2))
    bumped = [f.copy() for f in base]
    for c in range(3):
        bumped[c][:, :, m + 2] += 1.0                # 1-based plane m + 3
    out = {}
    for name, fields in (("base", base), ("bumped", bumped)):
        for tag, x in (("crossing", x_below), ("inside", m * s.dx + 1e-4)):
            ens = _one(s, 0.05, 2.0, (x, 3.0, 3.0), (0.5, 0.0, 0.0), (1.0, -1.0, 0.5))
            assert ens.advance(fields) == 0
            out[name, tag] = {k: ens.a[k].copy() for k in po.STATE_KEYS}
    assert out["base", "crossing"]["x"][0] > m * s.dx                  # the predictor did cross
    for k in po.STATE_KEYS:
        assert np.array_equal(out["base", "crossing"][k], out["bumped", "crossing"][k]), k
    assert not np.array_equal(out["base", "inside"]["u"], out["bumped", "inside"]["u"])


def _pair(s, dx):
    """Two spheroids of different size (so different inertia) closing on each other."""
    from gazpart_b200 import particles
    a = particles.draw(config.ParticleSpec(n=1, ar=1.5, b=0.05 / 1.5, st=1.0, seed=3), s)
    b = particles.draw(config.ParticleSpec(n=1, ar=2.0, b=0.08 / 2.0, st=1.0, seed=4), s)
    st = {k: np.concatenate([a[k], b[k]]) for k in a}
    st["x"][:] = [1.0, 1.0 + dx]
    st["y"][:] = [1.0, 1.02]
    st["z"][:] = [1.0, 1.01]
    st["u"][:] = [0.5, -0.5]
    st["v"][:] = 0.0
    st["w"][:] = 0.0
    for k in ("ox", "oy", "oz"):
        st[k][:] = [0.3, -0.2]
    q = np.array([[0.9, 0.3, 0.2, 0.1], [0.7, -0.1, 0.5, 0.3]])
    q /= np.linalg.norm(q, axis=1)[:, None]
    for c, k in enumerate(("qa", "qb", "qc", "qd")):
        st[k][:] = q[:, c]
    return st


def test_q8_first_particles_inertia_for_both():
    """Q8 (collision_response.f90:140-145): COLLISION_RESPONSE rotates particle 1's
    principal moments for both bodies, so the collision of a small and a large spheroid
    gives exactly the response computed with the home particle's inertia, not the
    other's."""
    s = config.Setup(nx=16, ny=16, nz=16, visc=0.05, dtime=1e-3)
    ens = po.Ensemble(s, _pair(s, 0.06))
    a = {k: v.copy() for k, v in ens.a.items()}
    e1, e2, cn, r1, r2 = (np.zeros(3) for _ in range(5))
    fl = C.c_int32()
    hit = po.lib().orc_pair_eval(C.byref(po.make_setup(s)), C.byref(ens.props()), C.byref(ens.state()),
                                 C.c_int64(0), C.c_int64(1), po.dptr(e1), po.dptr(e2), po.dptr(cn),
                                 po.dptr(r1), po.dptr(r2), C.byref(fl))
    assert hit == 1 and fl.value == 1
    res = ens.collide(prefilter=True)
    assert res["rc"] == 0 and list(res["home"]) == [0] and list(res["near"]) == [1]

    def response(i):
        ip = (a["ipxx"][i], a["ipyy"][i], a["ipzz"][i])
        q = [np.array([a[k][j] for k in ("qa", "qb", "qc", "qd")]) for j in (0, 1)]
        u = [np.array([a[k][j] for k in ("u", "v", "w")]) for j in (0, 1)]
        o = [np.array([a[k][j] for k in ("ox", "oy", "oz")]) for j in (0, 1)]
        return po.collision_response(s, ip, u[0], o[0], q[0], u[1], o[1], q[1], r1, r2, cn)

    got = [np.array([ens.a[k][j] for k in ("u", "v", "w")]) for j in (0, 1)]
    rc, u1, _, u2, _ = response(0)
    assert rc == 0 and np.array_equal(got[0], u1) and np.array_equal(got[1], u2)
    assert a["ipxx"][0] != a["ipxx"][1]
    rc, v1, _, v2, _ = response(1)
    assert not (np.array_equal(got[0], v1) and np.array_equal(got[1], v2))


def test_q9_energy_check_stops_inelastic_collisions():
    """Q9 (collision_response.f90:408-436): the response checks that kinetic energy is
    conserved to 1e-9 %, so any restitution below 1 stops the run (GP_EENERGY)."""
    ip = (1e-3, 1e-3, 1e-3)
    q = np.array([1.0, 0.0, 0.0, 0.0])
    n = np.array([1.0, 0.0, 0.0])
    args = (ip, [1.0, 0, 0], [0, 0, 0], q, [-1.0, 0, 0], [0, 0, 0], q, [0.1, 0, 0], [-0.1, 0, 0], n)
    elastic = config.Setup(nx=16, ny=16, nz=16, ecp=1.0, mup=0.0)
    rc, u1, _, u2, _ = po.collision_response(elastic, *args)
    assert rc == 0
    assert np.allclose(u1, [-1.0, 0, 0]) and np.allclose(u2, [1.0, 0, 0])   # equal masses swap
    inelastic = config.Setup(nx=16, ny=16, nz=16, ecp=0.9, mup=0.0)
    rc, *_ = po.collision_response(inelastic, *args)
    assert rc == 3                                          # GP_EENERGY


def test_q10_box_edge_from_the_major_semi_axis():
    """Q10 (collision_initiation.f90:50,69-75): DPMAX = 2 EMAJ and DXBOX =
    L / int(L / (2 DPMAX)), whatever the aspect ratio, so for oblate particles (APR < 1,
    b = EMAJ / APR > EMAJ) a box is narrower than two bounding diameters."""
    s = config.Setup(nx=16, ny=16, nz=16)
    g = po.OrcBoxGrid()
    emaj = 0.1
    po.lib().orc_collision_initiation(C.byref(po.make_setup(s)), C.c_double(emaj), C.byref(g))
    assert g.nxbox == int(L / (4 * emaj)) == 15
    assert g.dxbox == L / 15
    b_oblate = emaj / 0.2
    assert g.dxbox < 2 * (2 * b_oblate)


def test_q14_nan_starting_angle_reports_no_contact():
    """Q14 (ellipsoid_contact_detection.f90:77-87): the starting angles are
    asin(n_z) and acos(n_x / cos(asin(n_z))).  For a centre line in the x-z plane
    (n_y = 0) the ratio can round just above 1, acos gives NaN, every LM iterate stays
    NaN until maxfev, and the pair is not in contact, however deep the overlap.  Just
    out of that plane the same pairs are found in contact."""
    q1 = np.array([1.0, 0.0, 0.0, 0.0])
    q2 = np.array([0.9, 0.3, 0.2, 0.1])
    q2 /= np.linalg.norm(q2)
    nan_hits = 0
    for t in np.linspace(0.05, 1.5, 200):
        n = np.array([np.cos(t), 0.0, np.sin(t)])
        r = po.contact_detection(0.05, 1.5, 0.05, 1.5, np.zeros(3), q1, -0.05 * n, q2)
        if np.isnan(r["x"][0]):
            nan_hits += 1
            assert (r["flag"], r["info"], r["nfev"]) == (0, 5, 300)
            m = np.array([np.cos(t), 1e-3, np.sin(t)])
            m /= np.linalg.norm(m)
            r2 = po.contact_detection(0.05, 1.5, 0.05, 1.5, np.zeros(3), q1, -0.05 * m, q2)
            assert r2["flag"] == 1 and not np.isnan(r2["x"][0])
    assert nan_hits > 10


def test_q15_no_quaternion_renormalisation():
    """Q15 (adv_quaternion.f90:81): QUATERNION_INTEGRATION multiplies by a unit map
    quaternion and does not renormalise, so whatever norm q has is kept (the mixed
    form renormalises; the FP64 path keeps the reference's update)."""
    q = np.array([0.6, 0.48, 0.64, 0.0])
    q *= 1.1 / np.linalg.norm(q)
    om = np.array([3.1, -7.3, 11.9])
    for _ in range(100):
        q = po.quaternion_integration(q, om, 1.7e-3)
    assert abs(np.linalg.norm(q) - 1.1) < 1e-13


def test_q17_random_field_mode_takes_the_frozen_flow_2_boundary():
    """Q17 (adv_particle_new.f90:685-686): only FROZEN_FLOW 1-3 reach a boundary call,
    so the random-field mode runs as FROZEN_FLOW = 2, whose BOUNDARY_PARTICLE wraps
    every direction; the C ABI refuses FROZEN_FLOW 4 and above (it checks its arguments
    before it touches the device)."""
    import pytest
    from gazpart_b200 import api
    s = config.Setup(nx=16, ny=16, nz=16, visc=0.05, dtime=1e-3)
    assert s.frozen_flow == 2
    ens = _one(s, 0.02, 1.5, (3.0, 3.0, L - 1e-4), (0.0, 0.0, 0.5), (0.0, 0.0, 0.0))
    assert ens.advance(_quiet_field(s)) == 0
    assert 0.0 < ens.a["z"][0] < 1e-3                      # wrapped through z = L
    for bad in (0, 4):
        with pytest.raises(api.GPError) as e:
            api.Context(config.Setup(nx=16, ny=16, nz=16, frozen_flow=bad))
        assert e.value.code == 9                           # GP_EBADARG


def test_q19_x_equal_to_l_is_outside_the_box_grid():
    """Q19 (boundary_particle.f90:50; collision_detection_connectivity.f90:81-89): the
    wrap tests x > L strictly, so x == L stays, and its box index int(x / DXBOX) + 1 is
    NXBOX + 1: out of the grid."""
    s = config.Setup(nx=16, ny=16, nz=16)
    st = {k: np.zeros(2) for k in po.STATE_KEYS + po.PROP_KEYS}
    st["emaj"][:] = 0.05
    st["apr"][:] = 1.0
    ens = po.Ensemble(s, st)
    g = ens.boxgrid()
    rc, ijk = po.box_index(ens, g, x=[np.nextafter(L, 0.0), L], y=[1.0, 1.0], z=[1.0, 1.0])
    assert rc == 6 and ijk[0] > 0 and ijk[1] == 0          # ORC_EOUT_OF_GRID for x == L
