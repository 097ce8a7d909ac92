"""Live fluid: the reference's pseudo-spectral DNS step on the device (``gp_dns_*``).

In DNS mode (SOLVE_FLUID = 1) each cycle of the reference advances the particles
through the current field, then ADV_FLUID advances the field (adv_fluid.f90:1-271)
and FLUIDCOMM refreshes its ghost planes (main.f90:496-505).  :class:`Fluid` holds the
velocity on the device; :meth:`Fluid.couple` writes it into a particle context's field
slot, so the next particle step interpolates the live field instead of a frozen one::

    fluid = Fluid(setup)
    fluid.set_velocity(u, v, w)           # interior arrays [z][y][x]
    fluid.couple(ctx)
    for n in range(ncycle):
        ctx.adv_particle_ellp(n); ctx.collision(n, t)
        fluid.adv_fluid(n); fluid.couple(ctx)
"""
from __future__ import annotations

import ctypes as C
from typing import Tuple

import numpy as np

from . import _lib
from ._lib import check

ALIAS_NONE, ALIAS_SHARP, ALIAS_SMOOTH = 0, 1, 2
RTRUNC = 8.0 / 9.0          # meshing.f90:36, with ALIASCONTROL = 2 (meshing.f90:31)


class Fluid:
    def __init__(self, setup, aliascontrol: int = ALIAS_SMOOTH, rtrunc: float = RTRUNC):
        p = _lib.GPParams()
        p.nx, p.ny, p.nz = setup.nx, setup.ny, setup.nz
        p.lx, p.ly, p.lz = setup.lx, setup.ly, setup.lz
        p.visc, p.rhof, p.dtime = setup.visc, setup.rhof, setup.dtime
        self.shape = (setup.nz, setup.ny, setup.nx)
        self._h = C.c_void_p()
        check(_lib.lib().gp_dns_create(C.byref(p), int(aliascontrol), float(rtrunc), C.byref(self._h)),
              "gp_dns_create")

    def close(self) -> None:
        if self._h:
            _lib.lib().gp_dns_destroy(self._h)
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

    def _arrays(self, *arrs):
        out = []
        for a in arrs:
            a = np.ascontiguousarray(a, dtype=np.float64)
            if a.shape != self.shape:
                raise ValueError(f"expected shape {self.shape}, got {a.shape}")
            out.append(a)
        return out

    def set_velocity(self, u, v, w) -> None:
        """Interior arrays [z][y][x]: numpy on the host, or float64 CUDA tensors."""
        if all(hasattr(a, "is_cuda") and a.is_cuda for a in (u, v, w)):
            import torch
            ts = [a.to(torch.float64).contiguous() for a in (u, v, w)]
            if any(tuple(t.shape) != self.shape for t in ts):
                raise ValueError(f"expected shape {self.shape}")
            check(_lib.lib().gp_dns_set_velocity(self._h, *(t.data_ptr() for t in ts), 1), "gp_dns_set_velocity")
            torch.cuda.synchronize()
            return
        u, v, w = self._arrays(u, v, w)
        check(_lib.lib().gp_dns_set_velocity(self._h, u.ctypes.data, v.ctypes.data, w.ctypes.data, 0),
              "gp_dns_set_velocity")

    def velocity(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        u, v, w = (np.empty(self.shape) for _ in range(3))
        check(_lib.lib().gp_dns_get_velocity(self._h, u.ctypes.data, v.ctypes.data, w.ctypes.data, 0),
              "gp_dns_get_velocity")
        return u, v, w

    def vorticity(self) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        x, y, z = (np.empty(self.shape) for _ in range(3))
        check(_lib.lib().gp_dns_vorticity(self._h, x.ctypes.data, y.ctypes.data, z.ctypes.data, 0),
              "gp_dns_vorticity")
        return x, y, z

    def adv_fluid(self, ncycle: int = 0) -> None:
        """ADV_FLUID(NCYCLE): one step of the field."""
        check(_lib.lib().gp_adv_fluid(self._h, int(ncycle)), "gp_adv_fluid")

    def couple(self, ctx, field: int = 0, with_vorticity: bool = False) -> None:
        """The current velocity (and the spectral vorticity if asked) into ctx's field slot."""
        check(_lib.lib().gp_dns_couple(self._h, ctx._h, int(field), 1 if with_vorticity else 0), "gp_dns_couple")
