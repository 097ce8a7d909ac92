"""Host-side interface mirroring the reference routines on the hot path.

One :class:`Context` stands for the reference's module state of one particle class on
one GPU (mesh, physics, the frozen field, ``PART(:, IG)``).  Its methods carry the
reference routine names:

==========================  =========================================================
``adv_particle_ellp``       ``ADV_PARTICLE_ELLP(NCYCLE)``  adv_particle_new.f90:7
``collision``               ``COLLISION(NCYCLE, TIME)``     collision.f90:7
``interp_lag3``             ``INTERP_LAG3``                 interp_lag3.f90:11
``frozen_interp_lag3``      ``FROZEN_INTERP_LAG3``          frozen_interp_lag3.f90:11
``fluid_force_ellipsoid``   ``FLUID_FORCE_ELLIPSOID``       fluid_force_ellipsoid.f90:1
``fluid_torque_ellipsoid``  ``FLUID_TORQUE_ELLIPSOID``      fluid_torque_ellipsoid.f90:1
``quaternion_integration``  ``QUATERNION_INTEGRATION``      adv_quaternion.f90:1
``euler_integration``       ``EULER_INTEGRATION``           adv_angular_velocity.f90:1
``collision_box_connectivity`` ``COLLISION_BOX_CONNECTIVITY`` collision_box_connectivity.f90:7
``ellipsoid_contact_detection`` ``ellipsoid_contact_detection`` ellipsoid_contact_detection.f90:1
``collision_response``      ``COLLISION_RESPONSE``          collision_response.f90:1
==========================  =========================================================

Errors the reference handles with ``stop`` raise :class:`~gazpart_b200._lib.GPError`.
Every call goes to the CUDA library; nothing here computes particle physics.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import GPError, check

STATE_KEYS = ("x", "y", "z", "u", "v", "w", "qa", "qb", "qc", "qd", "ox", "oy", "oz")
PROP_KEYS = ("emaj", "apr", "rhop", "ipxx", "ipyy", "ipzz")
FLUID_KEYS = ("ufap", "vfap", "wfap", "vortx", "vorty", "vortz")
FIELD_KEYS = ("u", "v", "w", "vortx", "vorty", "vortz")


def _is_torch_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _ptr(a):
    """(pointer, on_device, keepalive) for a numpy array or a torch tensor."""
    if _is_torch_cuda(a):
        import torch
        assert a.dtype == torch.float64 and a.is_contiguous()
        return C.c_void_p(a.data_ptr()), 1, a
    if hasattr(a, "numpy") and not isinstance(a, np.ndarray):
        a = a.numpy()
    arr = np.ascontiguousarray(a, dtype=np.float64)
    return C.c_void_p(arr.ctypes.data), 0, arr


class Context:
    """A device context for one ensemble (particle class) and its frozen field."""

    def __init__(self, setup, precision: str = "fp64", store_fluid: bool = False, max_particles: int = 0):
        p = _lib.GPParams()
        p.nx, p.ny, p.nz = setup.nx, setup.ny, setup.nz
        p.lx, p.ly, p.lz = setup.lx, setup.ly, setup.lz
        p.visc, p.rhof, p.dtime, p.gravity = setup.visc, setup.rhof, setup.dtime, setup.gravity
        p.ecp, p.mup, p.ecw, p.muw = setup.ecp, setup.mup, setup.ecw, setup.muw
        p.periodicity = int(bool(setup.periodicity))
        p.wall_boundary = int(bool(setup.wall_boundary))
        p.interp_scheme = 3
        p.frozen_flow = int(getattr(setup, "frozen_flow", 2))
        p.precision = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
        p.store_fluid = int(bool(store_fluid))
        p.max_particles = int(max_particles)
        self.setup = setup
        self.precision = precision
        self.store_fluid = bool(store_fluid)
        self._h = C.c_void_p()
        check(_lib.lib().gp_ctx_create(C.byref(p), C.byref(self._h)), "gp_ctx_create")
        self.n = 0
        self._groups: Dict[int, int] = {}   # class -> polydisperse indices (gp_set_class_groups)

    # -- lifetime ------------------------------------------------------------
    def close(self) -> None:
        if self._h:
            _lib.lib().gp_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- status ---------------------------------------------------------------
    def status(self):
        code, fid = C.c_int32(), C.c_int64()
        check(_lib.lib().gp_status(self._h, C.byref(code), C.byref(fid)), "gp_status")
        return code.value, fid.value

    def collision_counters(self) -> Dict[str, int]:
        """Counters of the last collision phase (_lib.COUNTERS)."""
        v = (C.c_int64 * len(_lib.COUNTERS))()
        check(_lib.lib().gp_collision_counters(self._h, v), "gp_collision_counters")
        return dict(zip(_lib.COUNTERS, (int(x) for x in v)))

    # ---- statistics beside the step (gp_stats.cu) ----
    def set_class_groups(self, ig: int, idp: Optional[np.ndarray] = None, ngroups: Optional[int] = None) -> None:
        """Polydisperse index PART(I,IG)%IDP of each particle of class ig, in its own order
        (None: all 1)."""
        if idp is None:
            check(_lib.lib().gp_set_class_groups(self._h, int(ig), 1, None), "gp_set_class_groups")
            self._groups.pop(int(ig), None)
            return
        idp = np.ascontiguousarray(idp, dtype=np.int32)
        ng = int(idp.max()) if ngroups is None else int(ngroups)
        check(_lib.lib().gp_set_class_groups(self._h, int(ig), ng, idp.ctypes.data_as(_lib._ip)),
              "gp_set_class_groups")
        self._groups[int(ig)] = ng

    def stat_partfluid(self, ig: int = 1, sums: bool = False) -> np.ndarray:
        """STAT_PARTFLUID for class ig: MEAN_PARTFLUID(:, IG, IDP) per index, shape
        [ngroups, 36] (the last column the particle count), or the raw sums."""
        ng = self._groups.get(int(ig), 1)
        out = np.empty(ng * _lib.NSTAT_PARTFLUID)
        check(_lib.lib().gp_stat_partfluid(self._h, int(ig), out.ctypes.data_as(_lib._dp)), "gp_stat_partfluid")
        out = out.reshape(ng, _lib.NSTAT_PARTFLUID)
        if sums:
            return out
        mean = out / out[:, -1:]
        mean[:, -1] = out[:, -1]
        return mean

    def set_contact_tail(self, budget: int) -> None:
        """Solves running past `budget` evaluations finish in the inlined-solver kernel
        (0: none do); results are unchanged."""
        check(_lib.lib().gp_set_contact_tail(self._h, int(budget)), "gp_set_contact_tail")

    def contact_tail(self) -> int:
        b = C.c_int32()
        check(_lib.lib().gp_get_contact_tail(self._h, C.byref(b)), "gp_get_contact_tail")
        return b.value

    def set_contact_order(self, on: bool) -> None:
        """Hand the contact solves to the lanes in decreasing predicted length (the
        default) or in candidate-list order; results are unchanged."""
        check(_lib.lib().gp_set_contact_order(self._h, 1 if on else 0), "gp_set_contact_order")

    def contact_order(self) -> bool:
        v = C.c_int32()
        check(_lib.lib().gp_get_contact_order(self._h, C.byref(v)), "gp_get_contact_order")
        return bool(v.value)

    def set_gather_staging(self, mode: int) -> None:
        """Mixed gather: 0 stencil rows through L1, 1 each stencil box staged in shared
        memory by the TMA (one field for every class); results are unchanged."""
        check(_lib.lib().gp_set_gather_staging(self._h, int(mode)), "gp_set_gather_staging")

    def gather_staging(self) -> int:
        v = C.c_int32()
        check(_lib.lib().gp_get_gather_staging(self._h, C.byref(v)), "gp_get_gather_staging")
        return v.value

    def enable_collision_stats(self, on: bool = True) -> None:
        check(_lib.lib().gp_collision_stats_enable(self._h, 1 if on else 0), "gp_collision_stats_enable")

    def collision_stats(self, ig: int = 1, reset: bool = True):
        """MEAN_PART_COL(1:8, IDP1, IDP2) of class ig summed over the collision steps since
        the last reset: (array [ngroups, ngroups, 8], steps)."""
        ng = self._groups.get(int(ig), 1)
        out = np.empty(ng * ng * _lib.NSTAT_COLLISION)
        steps = C.c_int64()
        check(_lib.lib().gp_collision_stats(self._h, int(ig), out.ctypes.data_as(_lib._dp), C.byref(steps),
                                            1 if reset else 0), "gp_collision_stats")
        return out.reshape(ng, ng, _lib.NSTAT_COLLISION), steps.value

    def status_class(self) -> int:
        """Class (1-based) of the particle behind the first error; 0 if none."""
        ig = C.c_int32()
        check(_lib.lib().gp_status_class(self._h, C.byref(ig)), "gp_status_class")
        return ig.value

    def clear_status(self) -> None:
        check(_lib.lib().gp_clear_status(self._h), "gp_clear_status")

    def raise_status(self, where: str = "device") -> None:
        code, fid = self.status()
        if code:
            raise GPError(code, f"{where} (first id {fid})")

    def sync(self) -> None:
        check(_lib.lib().gp_sync(self._h), "gp_sync")

    # -- set-up ---------------------------------------------------------------
    def set_class(self, ig: int, idp: int, emaj: float, apr: float, rhop: float) -> None:
        check(_lib.lib().gp_set_class(self._h, ig, idp, emaj, apr, rhop), "gp_set_class")

    def set_field(self, comp: int, data, layout: str = "interior", ghost: str = "periodic") -> None:
        ptr, dev, keep = _ptr(data)
        lay = {"interior": _lib.LAYOUT_INTERIOR, "reference": _lib.LAYOUT_REFERENCE}[layout]
        gh = {"periodic": _lib.GHOST_PERIODIC, "zero": _lib.GHOST_ZERO}[ghost]
        check(_lib.lib().gp_set_field(self._h, comp, ptr, lay, gh, dev), "gp_set_field")

    def set_fields(self, fields: Dict[str, object], vorticity_ghost: str = "zero", slot: int = 0) -> None:
        """Velocity with periodic ghosts; vorticity ghosts as the reference leaves them
        (never exchanged, hence zero) unless ``vorticity_ghost='periodic'``.  ``slot``
        selects a resident field added by add_field."""
        for c, k in enumerate(FIELD_KEYS):
            ptr, dev, keep = _ptr(fields[k])
            gh = _lib.GHOST_PERIODIC if (c < 3 or vorticity_ghost == "periodic") else _lib.GHOST_ZERO
            check(_lib.lib().gp_set_field_slot(self._h, slot, c, ptr, _lib.LAYOUT_INTERIOR, gh, dev),
                  "gp_set_field_slot")

    def add_field(self, n: int, lbox: float = 2.0 * np.pi) -> int:
        """One more resident field of n^3 points on a periodic box of side lbox; returns its slot."""
        f = C.c_int32()
        check(_lib.lib().gp_add_field(self._h, n, n, n, lbox, lbox, lbox, C.byref(f)), "gp_add_field")
        return f.value

    def add_class(self, st: Dict[str, object], field: int = 0) -> int:
        """Admit one more class (host arrays) on field slot ``field``; returns its number."""
        n = int(np.asarray(st["x"]).shape[0])
        cat = {k: np.ascontiguousarray(np.asarray(st[k], dtype=np.float64)) for k in STATE_KEYS + PROP_KEYS}
        cols = (C.c_void_p * 13)(*[C.c_void_p(cat[k].ctypes.data) for k in STATE_KEYS])
        props = (C.c_void_p * 6)(*[C.c_void_p(cat[k].ctypes.data) for k in PROP_KEYS])
        ig = C.c_int32()
        check(_lib.lib().gp_add_class(self._h, field, n, cols, props, 0, C.byref(ig)), "gp_add_class")
        self._groups.pop(ig.value, None)
        self.n += n
        return ig.value

    def class_count(self, ig: int) -> int:
        n = C.c_int64()
        check(_lib.lib().gp_class_count(self._h, ig, C.byref(n)), "gp_class_count")
        return n.value

    def download_class(self, ig: int) -> Dict[str, np.ndarray]:
        n = self.class_count(ig)
        out = {k: np.empty(n) for k in STATE_KEYS}
        cols = (C.c_void_p * 13)(*[C.c_void_p(out[k].ctypes.data) for k in STATE_KEYS])
        check(_lib.lib().gp_download_class(self._h, ig, cols, 0), "gp_download_class")
        return out

    def remove_class(self, ig: int) -> Dict[str, np.ndarray]:
        """Retire class ig and return its final state."""
        n = self.class_count(ig)
        out = {k: np.empty(n) for k in STATE_KEYS}
        cols = (C.c_void_p * 13)(*[C.c_void_p(out[k].ctypes.data) for k in STATE_KEYS])
        check(_lib.lib().gp_remove_class(self._h, ig, cols, 0), "gp_remove_class")
        self._groups.pop(int(ig), None)
        self.n -= n
        return out

    def upload(self, st: Dict[str, object]) -> None:
        n = int(st["x"].shape[0])
        keep = []
        cols = (C.c_void_p * 13)()
        props = (C.c_void_p * 6)()
        dev = None
        for i, k in enumerate(STATE_KEYS):
            p, d, kk = _ptr(st[k])
            cols[i] = p
            keep.append(kk)
            dev = d if dev is None else dev
            if d != dev:
                raise ValueError("mixed host/device columns")
        for i, k in enumerate(PROP_KEYS):
            p, d, kk = _ptr(st[k])
            props[i] = p
            keep.append(kk)
            if d != dev:
                raise ValueError("mixed host/device columns")
        check(_lib.lib().gp_upload_state(self._h, n, cols, props, dev), "gp_upload_state")
        self._groups.clear()
        self.n = n
        self.class_counts = np.array([n], dtype=np.int64)

    def upload_classes(self, states) -> None:
        """Several classes (the reference's IG = 1..NIG) on this context's field, each with
        its own box and search grids, stepped together.  ``states``: one state dict per
        class (host numpy arrays).  download() returns the classes concatenated in this
        order; split_classes() cuts such a dict back into per-class dicts."""
        counts = np.array([int(st["x"].shape[0]) for st in states], dtype=np.int64)
        cat = {k: np.ascontiguousarray(np.concatenate([np.asarray(st[k], dtype=np.float64) for st in states]))
               for k in STATE_KEYS + PROP_KEYS}
        cols = (C.c_void_p * 13)(*[C.c_void_p(cat[k].ctypes.data) for k in STATE_KEYS])
        props = (C.c_void_p * 6)(*[C.c_void_p(cat[k].ctypes.data) for k in PROP_KEYS])
        check(_lib.lib().gp_upload_classes(self._h, len(states), counts.ctypes.data_as(_lib._i64p), cols, props, 0),
              "gp_upload_classes")
        self._groups.clear()
        self.n = int(counts.sum())
        self.class_counts = counts

    def split_classes(self, st: Dict[str, np.ndarray]):
        """Concatenated per-particle arrays -> one dict per class (upload_classes order)."""
        edges = np.concatenate([[0], np.cumsum(self.class_counts)])
        return [{k: v[edges[i]:edges[i + 1]] for k, v in st.items()} for i in range(len(self.class_counts))]

    def put_state(self, st: Dict[str, object]) -> None:
        """Overwrite the 13 state columns (properties unchanged), caller order."""
        keep, cols, dev = [], (C.c_void_p * 13)(), None
        for i, k in enumerate(STATE_KEYS):
            p, d, kk = _ptr(st[k])
            cols[i] = p
            keep.append(kk)
            dev = d
        check(_lib.lib().gp_put_state(self._h, self.n, cols, dev), "gp_put_state")

    def step_host(self, state: Dict[str, np.ndarray], out: Optional[Dict[str, np.ndarray]] = None
                  ) -> Dict[str, np.ndarray]:
        """One step of a host-resident ensemble (gp_step_host): the 13 state columns in
        (caller order), one step, the state out into `out` (default: `state` itself), with
        the copies overlapped with the step.  Arrays must be float64 and contiguous; pinned
        memory lets the copies run asynchronously."""
        out = state if out is None else out
        for d in (state, out):
            for k in STATE_KEYS:
                a = d[k]
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
                        and a.shape == (self.n,)):
                    raise ValueError(f"{k}: expected a contiguous float64 array of {self.n} values")
        cin = (C.c_void_p * 13)(*[C.c_void_p(state[k].ctypes.data) for k in STATE_KEYS])
        cout = (C.c_void_p * 13)(*[C.c_void_p(out[k].ctypes.data) for k in STATE_KEYS])
        check(_lib.lib().gp_step_host(self._h, self.n, cin, cout), "gp_step_host")
        return out

    def download_into(self, out: Dict[str, np.ndarray]) -> None:
        """Download the state columns into preallocated (e.g. pinned) float64 arrays."""
        cols = (C.c_void_p * 13)(*[C.c_void_p(out[k].ctypes.data) for k in STATE_KEYS])
        check(_lib.lib().gp_download_state(self._h, self.n, cols, None, 0), "gp_download_state")

    def step_timed(self, nsteps: int):
        """Run nsteps as one graph with device timestamps between the phases.

        Returns (total_ms, {phase: ms per step}, kernels per step); the phases are
        _lib.PHASES (gather, integrate, bin, search, contact, response)."""
        t, k = C.c_float(), C.c_int32()
        ph = (C.c_float * len(_lib.PHASES))()
        check(_lib.lib().gp_step_timed(self._h, nsteps, C.byref(t), ph, C.byref(k)), "gp_step_timed")
        return t.value, dict(zip(_lib.PHASES, (float(v) for v in ph))), k.value

    def autotune(self) -> Dict[str, int]:
        """Pick the launch grids on the resident ensemble (state restored afterwards)."""
        g = (C.c_int32 * (len(_lib.TUNABLES) + 1))()
        check(_lib.lib().gp_autotune(self._h, g), "gp_autotune")
        out = dict(zip(_lib.TUNABLES, (int(v) for v in g)))
        out["overlap_gather"] = bool(g[len(_lib.TUNABLES)])
        out["speculative_integrate"] = g[len(_lib.TUNABLES)] == 2
        out["contact_tail"] = self.contact_tail()
        out["gather_staging"] = self.gather_staging()
        return out

    def set_launch(self, grids: Dict[str, int]) -> None:
        """Launch grids and overlap choices as autotune() reports them
        (speculative_integrate implies overlap_gather)."""
        over = 2 if grids.get("speculative_integrate", False) else int(bool(grids.get("overlap_gather", False)))
        g = (C.c_int32 * (len(_lib.TUNABLES) + 1))(*[int(grids[k]) for k in _lib.TUNABLES], over)
        check(_lib.lib().gp_set_launch(self._h, g), "gp_set_launch")
        if "contact_tail" in grids:
            self.set_contact_tail(int(grids["contact_tail"]))
        if "gather_staging" in grids:
            self.set_gather_staging(int(grids["gather_staging"]))

    def download(self, fluid: bool = False) -> Dict[str, np.ndarray]:
        out = {k: np.empty(self.n) for k in STATE_KEYS}
        cols = (C.c_void_p * 13)(*[C.c_void_p(out[k].ctypes.data) for k in STATE_KEYS])
        fl = None
        if fluid:
            for k in FLUID_KEYS:
                out[k] = np.empty(self.n)
            fl = (C.c_void_p * 6)(*[C.c_void_p(out[k].ctypes.data) for k in FLUID_KEYS])
        check(_lib.lib().gp_download_state(self._h, self.n, cols, fl, 0), "gp_download_state")
        return out

    # -- hot path -------------------------------------------------------------
    def adv_particle_ellp(self, ncycle: int = 0) -> None:
        check(_lib.lib().gp_adv_particle_ellp(self._h, ncycle), "gp_adv_particle_ellp")

    def collision(self, ncycle: int = 0, time: float = 0.0):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(_lib.lib().gp_collision(self._h, ncycle, time, C.byref(a), C.byref(b), C.byref(c)), "gp_collision")
        return {"n_near": a.value, "n_contact": b.value, "n_coll": c.value}

    def step(self, nsteps: int = 1) -> None:
        check(_lib.lib().gp_step(self._h, nsteps), "gp_step")

    def collision_pairs(self):
        cnt = C.c_int64()
        check(_lib.lib().gp_collision_pairs(self._h, 0, None, None, C.byref(cnt)), "gp_collision_pairs")
        n = cnt.value
        home = np.zeros(max(n, 1), dtype=np.int32)
        near = np.zeros(max(n, 1), dtype=np.int32)
        check(_lib.lib().gp_collision_pairs(self._h, n, home.ctypes.data_as(_lib._ip), near.ctypes.data_as(_lib._ip),
                                            C.byref(cnt)), "gp_collision_pairs")
        return home[:n], near[:n]

    def set_pair_capacity(self, cap_pairs: int, cap_coll: int) -> None:
        """Sizes of the candidate-pair and colliding-pair buffers (gp_set_pair_capacity);
        a step that outgrows them grows them and runs again, with the same results."""
        check(_lib.lib().gp_set_pair_capacity(self._h, int(cap_pairs), int(cap_coll)), "gp_set_pair_capacity")

    def pair_capacity(self):
        a, b = C.c_int64(), C.c_int64()
        check(_lib.lib().gp_pair_capacity(self._h, C.byref(a), C.byref(b)), "gp_pair_capacity")
        return a.value, b.value

    def collision_box_connectivity(self):
        nbox = C.c_int32()
        dims = np.zeros(3, dtype=np.int32)
        geom = np.zeros(6)
        check(_lib.lib().gp_collision_box_connectivity(self._h, C.byref(nbox), None, None,
                                                       dims.ctypes.data_as(_lib._ip), geom.ctypes.data_as(_lib._dp)),
              "gp_collision_box_connectivity")
        ncon = np.zeros(nbox.value, dtype=np.int32)
        con = np.zeros(nbox.value * 27, dtype=np.int32)
        check(_lib.lib().gp_collision_box_connectivity(self._h, C.byref(nbox), ncon.ctypes.data_as(_lib._ip),
                                                       con.ctypes.data_as(_lib._ip), None, None),
              "gp_collision_box_connectivity")
        return {"dims": dims, "geom": geom, "ncon": ncon, "con": con}

    # -- per-routine drop-ins ---------------------------------------------------
    def interp_lag3(self, comp: int, x, y, z):
        if _is_torch_cuda(x):
            import torch
            out = torch.empty_like(x)
            check(_lib.lib().gp_interp_lag3(self._h, comp, x.numel(), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                            C.c_void_p(z.data_ptr()), C.c_void_p(out.data_ptr()), 1), "gp_interp_lag3")
            return out
        x, y, z = (np.ascontiguousarray(t, dtype=np.float64) for t in (x, y, z))
        out = np.empty_like(x)
        check(_lib.lib().gp_interp_lag3(self._h, comp, x.size, C.c_void_p(x.ctypes.data), C.c_void_p(y.ctypes.data),
                                        C.c_void_p(z.ctypes.data), C.c_void_p(out.ctypes.data), 0), "gp_interp_lag3")
        return out

    def frozen_interp_lag3(self, xain, yain, zain, uain, x, y, z):
        """uain: numpy (NZ, NY, NX) == Fortran (NX, NY, NZ)."""
        nz, ny, nx = uain.shape
        arrs = [np.ascontiguousarray(t, dtype=np.float64) for t in (xain, yain, zain, uain, x, y, z)]
        out = np.empty_like(arrs[4])
        dp = [a.ctypes.data_as(_lib._dp) for a in arrs]
        check(_lib.lib().gp_frozen_interp_lag3(self._h, dp[0], dp[1], dp[2], nx, ny, nz, dp[3], arrs[4].size, dp[4],
                                               dp[5], dp[6], out.ctypes.data_as(_lib._dp)), "gp_frozen_interp_lag3")
        return out

    def fluid_force_ellipsoid(self, ig, idp, up, uf, quat):
        ig = np.ascontiguousarray(ig, dtype=np.int32).reshape(-1)
        idp = np.ascontiguousarray(idp, dtype=np.int32).reshape(-1)
        n = ig.size
        up, uf, q = (np.ascontiguousarray(a, dtype=np.float64).reshape(n, -1) for a in (up, uf, quat))
        fd, fl = np.empty((n, 3)), np.empty((n, 3))
        a = [C.c_void_p(t.ctypes.data) for t in (ig, idp, up, uf, q, fd, fl)]
        check(_lib.lib().gp_fluid_force_ellipsoid_batch(self._h, n, *a, 0), "gp_fluid_force_ellipsoid")
        return fd, fl

    def fluid_torque_ellipsoid(self, ig, idp, omega, quat, part_up, part_ufap, part_vort):
        ig = np.ascontiguousarray(ig, dtype=np.int32).reshape(-1)
        idp = np.ascontiguousarray(idp, dtype=np.int32).reshape(-1)
        n = ig.size
        arrs = [np.ascontiguousarray(a, dtype=np.float64).reshape(n, -1)
                for a in (omega, quat, part_up, part_ufap, part_vort)]
        tp, tr = np.empty((n, 3)), np.empty((n, 3))
        a = [C.c_void_p(t.ctypes.data) for t in (ig, idp, *arrs, tp, tr)]
        check(_lib.lib().gp_fluid_torque_ellipsoid_batch(self._h, n, *a, 0), "gp_fluid_torque_ellipsoid")
        return tp, tr

    def quaternion_integration(self, quat, omega, dt: float):
        q = np.ascontiguousarray(quat, dtype=np.float64).reshape(-1, 4).copy()
        om = np.ascontiguousarray(omega, dtype=np.float64).reshape(-1, 3)
        check(_lib.lib().gp_quaternion_integration_batch(self._h, q.shape[0], C.c_void_p(q.ctypes.data),
                                                         C.c_void_p(om.ctypes.data), dt, 0), "gp_quaternion_integration")
        return q

    def euler_integration(self, ig: int, idp: int, omega):
        ox, oy, oz = (C.c_double(float(v)) for v in omega)
        check(_lib.lib().gp_euler_integration(self._h, ig, idp, C.byref(ox), C.byref(oy), C.byref(oz)),
              "gp_euler_integration")
        return np.array([ox.value, oy.value, oz.value])

    def ellipsoid_contact_detection(self, shapes, centres, quats):
        """shapes (n,4) emaj1 apr1 emaj2 apr2; centres (n,6); quats (n,8)."""
        s = np.ascontiguousarray(shapes, dtype=np.float64).reshape(-1, 4)
        n = s.shape[0]
        c = np.ascontiguousarray(centres, dtype=np.float64).reshape(n, 6)
        q = np.ascontiguousarray(quats, dtype=np.float64).reshape(n, 8)
        flag = np.empty(n, dtype=np.int32)
        e1, e2, cn = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        a = [C.c_void_p(t.ctypes.data) for t in (s, c, q, flag, e1, e2, cn)]
        check(_lib.lib().gp_ellipsoid_contact_detection_batch(self._h, n, *a, 0), "ellipsoid_contact_detection")
        return flag, e1, e2, cn

    def collision_response(self, ig: int, idp: int, part1, part2, r1, r2, normal):
        p1 = np.ascontiguousarray(part1, dtype=np.float64).copy()
        p2 = np.ascontiguousarray(part2, dtype=np.float64).copy()
        a = [np.ascontiguousarray(t, dtype=np.float64) for t in (r1, r2, normal)]
        rc = _lib.lib().gp_collision_response(self._h, ig, idp, p1.ctypes.data_as(_lib._dp),
                                              p2.ctypes.data_as(_lib._dp), *[t.ctypes.data_as(_lib._dp) for t in a])
        return rc, p1, p2
