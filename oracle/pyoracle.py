"""ctypes binding of the CPU restatement (``libgazpart_oracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py``, never by the product package.  PARITY UNPINNED
against the reference binary; see ``gazpart_oracle.h``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgazpart_oracle.so")
# the same restatement with libm's sin/cos/asin/acos in the contact solve, as the
# reference computes them (the default build shares its trigonometry with the device)
LIB_PATHS = {"shared": LIB_PATH, "libm": os.path.join(HERE, "libgazpart_oracle_libm.so")}

STATE_KEYS = ("x", "y", "z", "u", "v", "w", "qa", "qb", "qc", "qd", "ox", "oy", "oz")
AUX_KEYS = ("ufap", "vfap", "wfap", "vortx", "vorty", "vortz")
PROP_KEYS = ("emaj", "apr", "rhop", "ipxx", "ipyy", "ipzz")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class OrcSetup(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("visc", C.c_double), ("rhof", C.c_double), ("ppi", C.c_double),
                ("dtime", C.c_double), ("gravity", C.c_double),
                ("ecp", C.c_double), ("mup", C.c_double), ("ecw", C.c_double), ("muw", C.c_double),
                ("periodicity", C.c_int32), ("wall_boundary", C.c_int32), ("frozen_flow", C.c_int32)]


class OrcProps(C.Structure):
    _fields_ = [(k, _dp) for k in PROP_KEYS]


class OrcState(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(k, _dp) for k in STATE_KEYS + AUX_KEYS]


class OrcBoxGrid(C.Structure):
    _fields_ = [("nxbox", C.c_int32), ("nybox", C.c_int32), ("nzbox", C.c_int32), ("nbox", C.c_int32),
                ("dxbox", C.c_double), ("dybox", C.c_double), ("dzbox", C.c_double),
                ("xminbox", C.c_double), ("yminbox", C.c_double), ("zminbox", C.c_double),
                ("xmaxbox", C.c_double), ("ymaxbox", C.c_double), ("zmaxbox", C.c_double),
                ("delta_coll", C.c_double)]


_libs = {}


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(variant: str = "shared"):
    """The oracle library: "shared" (contact-solve trigonometry shared with the device)
    or "libm" (libm's, as the reference calls it)."""
    if variant not in _libs:
        path = LIB_PATHS[variant]
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_enorm.restype = C.c_double
        L.orc_fmargin.restype = C.c_double
        L.orc_detect_pairs.restype = C.c_int64
        L.orc_contact_detection.restype = C.c_int32
        L.orc_pair_eval.restype = C.c_int32
        _libs[variant] = L
    return _libs[variant]


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_ip)


def make_setup(s) -> OrcSetup:
    """OrcSetup from a gazpart_b200.config.Setup (or any object with the same fields)."""
    return OrcSetup(s.nx, s.ny, s.nz, s.lx, s.ly, s.lz, s.dx, s.dy, s.dz, s.visc, s.rhof,
                    4.0 * np.arctan(1.0), s.dtime, s.gravity, s.ecp, s.mup, s.ecw, s.muw,
                    int(bool(s.periodicity)), int(bool(s.wall_boundary)), int(getattr(s, "frozen_flow", 2)))


class Ensemble:
    """Numpy-backed particle state + properties driven through the oracle."""

    def __init__(self, setup, arrays: Dict[str, np.ndarray], variant: str = "shared"):
        self.setup = setup
        self.L = lib(variant)
        self.n = int(arrays["x"].shape[0])
        self.a = {}
        for k in STATE_KEYS + PROP_KEYS:
            self.a[k] = np.ascontiguousarray(arrays[k], dtype=np.float64).copy()
        for k in AUX_KEYS:
            self.a[k] = np.zeros(self.n)
        self._keep = []

    def props(self) -> OrcProps:
        return OrcProps(*[dptr(self.a[k]) for k in PROP_KEYS])

    def state(self) -> OrcState:
        return OrcState(self.n, *[dptr(self.a[k]) for k in STATE_KEYS + AUX_KEYS])

    def advance(self, fields_ref: Sequence[np.ndarray], nthreads: int = 1) -> int:
        """One ADV_PARTICLE_ELLP step; fields in the reference ghosted layout."""
        arr = (_dp * 6)(*[dptr(f) for f in fields_ref])
        s = make_setup(self.setup)
        st = self.state()
        eid = C.c_int64(-1)
        rc = self.L.orc_adv_particle_ellp(C.byref(s), C.byref(self.props()), arr, C.byref(st),
                                         C.c_int32(nthreads), C.byref(eid))
        self.last_err_id = eid.value
        return rc

    def boxgrid(self) -> OrcBoxGrid:
        g = OrcBoxGrid()
        s = make_setup(self.setup)
        self.L.orc_collision_initiation(C.byref(s), C.c_double(float(self.a["emaj"].max())), C.byref(g))
        return g

    def connectivity(self, g: OrcBoxGrid):
        ncon = np.zeros(g.nbox, dtype=np.int32)
        con = np.zeros(g.nbox * 27, dtype=np.int32)
        self.L.orc_box_connectivity(C.byref(g), C.c_int32(int(bool(self.setup.periodicity))),
                                   iptr(ncon), iptr(con))
        return ncon, con

    def collide(self, prefilter: bool = True, nthreads: int = 1, cap: int = 1 << 22,
                grid=None):
        g = self.boxgrid() if grid is None else grid
        ncon, con = self.connectivity(g)
        s = make_setup(self.setup)
        st = self.state()
        home = np.zeros(cap, dtype=np.int32)
        near = np.zeros(cap, dtype=np.int32)
        ncoll, ncand, ncont, eid = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        rc = self.L.orc_collision(C.byref(s), C.byref(self.props()), C.byref(g), iptr(ncon), iptr(con),
                                 C.byref(st), C.c_int32(int(prefilter)), C.c_int32(nthreads),
                                 C.c_int64(cap), iptr(home), iptr(near), C.byref(ncoll),
                                 C.byref(ncand), C.byref(ncont), C.byref(eid))
        k = min(ncoll.value, cap)
        return {"rc": rc, "home": home[:k].copy(), "near": near[:k].copy(),
                "n_coll": ncoll.value, "n_candidates": ncand.value, "n_contacts": ncont.value,
                "err_id": eid.value}

    def collide_stats(self, group: Optional[np.ndarray] = None, ngroups: int = 1, prefilter: bool = True,
                      grid=None):
        """COLLISION with the collision statistics of COLLISION_INTERACTION (serial walk):
        returns (rc, stats[ngroups, ngroups, 8], n_coll)."""
        g = self.boxgrid() if grid is None else grid
        ncon, con = self.connectivity(g)
        s = make_setup(self.setup)
        st = self.state()
        out = np.zeros(ngroups * ngroups * 8)
        gp = None
        if group is not None:
            group = np.ascontiguousarray(group, dtype=np.int32)
            gp = iptr(group)
        ncoll, eid = C.c_int64(), C.c_int64()
        rc = self.L.orc_collision_stats(C.byref(s), C.byref(self.props()), C.byref(g), iptr(ncon), iptr(con),
                                       C.byref(st), C.c_int32(int(prefilter)), gp, C.c_int32(ngroups),
                                       dptr(out), C.byref(ncoll), C.byref(eid))
        return rc, out.reshape(ngroups, ngroups, 8), ncoll.value

    def stat_partfluid(self, group: Optional[np.ndarray] = None, ngroups: int = 1) -> np.ndarray:
        """STAT_PARTFLUID sums per index over the particles in order: [ngroups, 36], the
        last entry the count (needs the fluid values of a step, self.a["ufap"]..)."""
        s = make_setup(self.setup)
        st = self.state()
        out = np.zeros(ngroups * 36)
        gp = None
        if group is not None:
            group = np.ascontiguousarray(group, dtype=np.int32)
            gp = iptr(group)
        self.L.orc_stat_partfluid(C.byref(s), C.byref(self.props()), C.byref(st), gp, C.c_int32(ngroups), dptr(out))
        return out.reshape(ngroups, 36)


def interp_lag3(setup, field_ref: np.ndarray, x, y, z) -> np.ndarray:
    s = make_setup(setup)
    x, y, z = (np.ascontiguousarray(t, dtype=np.float64) for t in (x, y, z))
    out = np.zeros_like(x)
    lib().orc_interp_lag3(C.byref(s), dptr(np.ascontiguousarray(field_ref)), C.c_int64(x.size),
                          dptr(x), dptr(y), dptr(z), dptr(out))
    return out


def frozen_interp_lag3(xain, yain, zain, uain, x, y, z) -> np.ndarray:
    """uain: numpy (NZ, NY, NX) C-order == Fortran (NX, NY, NZ)."""
    nz, ny, nx = uain.shape
    x, y, z = (np.ascontiguousarray(t, dtype=np.float64) for t in (x, y, z))
    out = np.zeros_like(x)
    lib().orc_frozen_interp_lag3(dptr(np.ascontiguousarray(xain, dtype=np.float64)),
                                 dptr(np.ascontiguousarray(yain, dtype=np.float64)),
                                 dptr(np.ascontiguousarray(zain, dtype=np.float64)),
                                 C.c_int32(nx), C.c_int32(ny), C.c_int32(nz),
                                 dptr(np.ascontiguousarray(uain, dtype=np.float64)), C.c_int64(x.size),
                                 dptr(x), dptr(y), dptr(z), dptr(out))
    return out


def _v(vals, n):
    return np.ascontiguousarray(np.asarray(vals, dtype=np.float64).reshape(n))


def fluid_force(setup, emaj, apr, rhop, up, uf, q):
    s = make_setup(setup)
    fd, fl = np.zeros(3), np.zeros(3)
    q = _v(q, 4)
    rc = lib().orc_fluid_force(C.byref(s), C.c_double(emaj), C.c_double(apr), C.c_double(rhop),
                               C.c_double(up[0]), C.c_double(up[1]), C.c_double(up[2]),
                               C.c_double(uf[0]), C.c_double(uf[1]), C.c_double(uf[2]),
                               dptr(q), dptr(fd), dptr(fl))
    return rc, fd, fl


def fluid_torque(setup, emaj, apr, rhop, up_n, uf, vort, om, q):
    s = make_setup(setup)
    tp, tr = np.zeros(3), np.zeros(3)
    q = _v(q, 4)
    args = [C.c_double(float(t)) for t in (*up_n, *uf, *vort, *om)]
    rc = lib().orc_fluid_torque(C.byref(s), C.c_double(emaj), C.c_double(apr), C.c_double(rhop),
                                *args, dptr(q), dptr(tp), dptr(tr))
    return rc, tp, tr


def quaternion_integration(q, om, dt):
    q = _v(q, 4).copy()
    lib().orc_quaternion_integration(dptr(q), C.c_double(om[0]), C.c_double(om[1]), C.c_double(om[2]),
                                     C.c_double(dt))
    return q


def euler_integration(ip, om, dt):
    ox, oy, oz = C.c_double(om[0]), C.c_double(om[1]), C.c_double(om[2])
    lib().orc_euler_integration(C.c_double(ip[0]), C.c_double(ip[1]), C.c_double(ip[2]), C.c_double(dt),
                                C.byref(ox), C.byref(oy), C.byref(oz))
    return np.array([ox.value, oy.value, oz.value])


def transform_vec(v, q):
    v = _v(v, 3).copy()
    lib().orc_transform_vec(dptr(v), dptr(_v(q, 4)))
    return v


def contact_detection(emaj1, apr1, emaj2, apr2, b1, q1, b2, q2, variant: str = "shared"):
    e1, e2, cn, xo = np.zeros(3), np.zeros(3), np.zeros(3), np.zeros(2)
    info, nfev = C.c_int32(), C.c_int32()
    flag = lib(variant).orc_contact_detection(C.c_double(emaj1), C.c_double(apr1), C.c_double(emaj2),
                                       C.c_double(apr2), dptr(_v(b1, 3)), dptr(_v(q1, 4)),
                                       dptr(_v(b2, 3)), dptr(_v(q2, 4)), dptr(e1), dptr(e2),
                                       dptr(cn), dptr(xo), C.byref(info), C.byref(nfev))
    return {"flag": int(flag), "ept1": e1, "ept2": e2, "cnormal": cn, "x": xo,
            "info": info.value, "nfev": nfev.value}


def fmargin(emaj, apr, point, center, q) -> float:
    return lib().orc_fmargin(C.c_double(emaj), C.c_double(apr), dptr(_v(point, 3)),
                             dptr(_v(center, 3)), dptr(_v(q, 4)))


def collision_response(setup, ip, u1, o1, q1, u2, o2, q2, r1, r2, n):
    s = make_setup(setup)
    u1, o1, u2, o2 = (_v(t, 3).copy() for t in (u1, o1, u2, o2))
    rc = lib().orc_collision_response(C.byref(s), C.c_double(ip[0]), C.c_double(ip[1]),
                                      C.c_double(ip[2]), dptr(u1), dptr(o1), dptr(_v(q1, 4)),
                                      dptr(u2), dptr(o2), dptr(_v(q2, 4)), dptr(_v(r1, 3)),
                                      dptr(_v(r2, 3)), dptr(_v(n, 3)))
    return rc, u1, o1, u2, o2


def wall_boundary_condition(setup, emaj, apr, pos, q):
    s = make_setup(setup)
    wn, arm = np.zeros(3), np.zeros(3)
    dx = C.c_double(0.0)
    isect = C.c_int32(0)
    rc = lib().orc_wall_boundary_condition(C.byref(s), C.c_double(emaj), C.c_double(apr),
                                           C.c_double(pos[0]), C.c_double(pos[1]), C.c_double(pos[2]),
                                           dptr(_v(q, 4)), dptr(wn), dptr(arm), C.byref(dx), C.byref(isect))
    return rc, wn, arm, dx.value, isect.value


def wall_rebound(setup, ip, u, om, q, arm, wn):
    s = make_setup(setup)
    vals = [C.c_double(float(t)) for t in (*u, *om)]
    rc = lib().orc_wall_rebound(C.byref(s), C.c_double(ip[0]), C.c_double(ip[1]), C.c_double(ip[2]),
                                *[C.byref(v) for v in vals], dptr(_v(q, 4)), dptr(_v(arm, 3)),
                                dptr(_v(wn, 3)))
    return rc, np.array([v.value for v in vals[:3]]), np.array([v.value for v in vals[3:]])


def enorm(x) -> float:
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().orc_enorm(C.c_int32(x.size), dptr(x))


def detect_pairs(ens: Ensemble, cap: Optional[int] = None):
    g = ens.boxgrid()
    ncon, con = ens.connectivity(g)
    a = ens.a
    n = lib().orc_detect_pairs(C.byref(g), iptr(ncon), iptr(con), C.c_int64(ens.n), dptr(a["x"]),
                               dptr(a["y"]), dptr(a["z"]), C.c_int64(0), None, None)
    if n < 0:
        raise RuntimeError("particle outside the collision grid")
    cap = n if cap is None else cap
    home = np.zeros(max(cap, 1), dtype=np.int32)
    near = np.zeros(max(cap, 1), dtype=np.int32)
    lib().orc_detect_pairs(C.byref(g), iptr(ncon), iptr(con), C.c_int64(ens.n), dptr(a["x"]),
                           dptr(a["y"]), dptr(a["z"]), C.c_int64(cap), iptr(home), iptr(near))
    return home[:min(n, cap)], near[:min(n, cap)]


def box_index(ens: Ensemble, g: OrcBoxGrid, x=None, y=None, z=None):
    a = ens.a
    x = a["x"] if x is None else np.ascontiguousarray(x, dtype=np.float64)
    y = a["y"] if y is None else np.ascontiguousarray(y, dtype=np.float64)
    z = a["z"] if z is None else np.ascontiguousarray(z, dtype=np.float64)
    ijk = np.zeros(x.size, dtype=np.int32)
    eid = C.c_int64()
    rc = lib().orc_box_index(C.byref(g), C.c_int64(x.size), dptr(x), dptr(y), dptr(z), iptr(ijk), C.byref(eid))
    return rc, ijk
