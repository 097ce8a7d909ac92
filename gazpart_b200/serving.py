"""Serving: tracking jobs streamed into one context with resident fields.

``serve`` hands a job list to the library's serving loop (``gp_serve``): jobs arrive at
their times, are admitted in arrival order against an HBM budget, and every loop
iteration advances and collides all running jobs in the same launches; finished jobs
leave with their final state.  Each job is one class of the context (its own search and
box grids, collisions only within itself), so a job's result does not depend on which
others shared its steps.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import time
from typing import Dict, List, Optional

import numpy as np

from . import _lib
from .api import PROP_KEYS, STATE_KEYS, Context, check

# Device bytes one resident particle costs: two pool buffers (13 state + 10 constant
# doubles, id, class), the six interpolated field values, the search arrays (cell,
# order, position, radius, packed float4, axis, semi-axes, box key, class, id), the
# matching words, its share of the pair and contact buffers, and the contact queue's
# order (the particle's record of its last solves, a pair slot's order and bin).
BYTES_PER_PARTICLE = 2 * (23 * 8 + 8) + 6 * 8 + (4 + 4 + 32 + 16 + 24 + 16 + 8 + 8) + 17 + 24 + 26 + 4 + 5


class GPJob(C.Structure):
    _fields_ = [("field", C.c_int32), ("steps", C.c_int32), ("n", C.c_int64), ("arrival_s", C.c_double),
                ("cols", C.POINTER(C.c_void_p)), ("props", C.POINTER(C.c_void_p)),
                ("admitted_s", C.c_double), ("done_s", C.c_double), ("status", C.c_int32), ("pad", C.c_int32)]


@dataclasses.dataclass
class Job:
    state: Dict[str, np.ndarray]     # initial state and properties (host arrays)
    steps: int
    arrival_s: float = 0.0
    field: int = 0
    # results
    result: Optional[Dict[str, np.ndarray]] = None
    admitted_s: float = -1.0
    done_s: float = -1.0
    status: int = 0

    @property
    def n(self) -> int:
        return int(self.state["x"].shape[0])

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s


def serve(ctx: Context, jobs: List[Job], hbm_budget: float, bytes_per_particle: float = BYTES_PER_PARTICLE):
    """Run the job stream; fills each job's result and times.  Returns a summary dict."""
    keep = []
    arr = (GPJob * len(jobs))()
    for i, j in enumerate(jobs):
        cols = {k: np.ascontiguousarray(np.array(j.state[k], dtype=np.float64)) for k in STATE_KEYS}
        props = {k: np.ascontiguousarray(np.asarray(j.state[k], dtype=np.float64)) for k in PROP_KEYS}
        cp = (C.c_void_p * 13)(*[C.c_void_p(cols[k].ctypes.data) for k in STATE_KEYS])
        pp = (C.c_void_p * 6)(*[C.c_void_p(props[k].ctypes.data) for k in PROP_KEYS])
        keep.append((cols, props, cp, pp))
        arr[i].field, arr[i].steps, arr[i].n, arr[i].arrival_s = j.field, j.steps, j.n, j.arrival_s
        arr[i].cols = C.cast(cp, C.POINTER(C.c_void_p))
        arr[i].props = C.cast(pp, C.POINTER(C.c_void_p))
    work = C.c_int64()
    t0 = time.perf_counter()
    check(_lib.lib().gp_serve(ctx._h, C.cast(arr, C.c_void_p), len(jobs), float(hbm_budget), float(bytes_per_particle),
                              C.byref(work)), "gp_serve")
    wall = time.perf_counter() - t0
    for i, j in enumerate(jobs):
        j.admitted_s, j.done_s, j.status = arr[i].admitted_s, arr[i].done_s, arr[i].status
        j.result = {k: keep[i][0][k] for k in STATE_KEYS}
    ok = [j for j in jobs if j.status == 0]
    lat = np.array([j.latency_s for j in ok]) if ok else np.array([np.nan])
    return {"wall_s": wall, "particle_steps": int(work.value), "particle_steps_per_s": work.value / wall,
            "jobs": len(jobs), "failed": len(jobs) - len(ok),
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "max_concurrent": max_concurrent(jobs)}


def max_concurrent(jobs: List[Job]) -> int:
    """Largest number of jobs resident at once (from the admission and completion times)."""
    ev = sorted([(j.admitted_s, 1) for j in jobs if j.admitted_s >= 0] +
                [(j.done_s, -1) for j in jobs if j.done_s >= 0], key=lambda e: (e[0], e[1]))
    cur = best = 0
    for _, d in ev:
        cur += d
        best = max(best, cur)
    return best
