"""CPU restatement of the reference's pseudo-spectral DNS step (numpy FFTs).

TEST INFRASTRUCTURE ONLY: the oracle of the device solver in
``gazpart_b200/csrc/gp_dns.cu``; nothing in the product imports it.

PARITY UNPINNED against the reference itself (its Fortran cannot be built here).  It is
pinned instead by known answers: a field with no nonlinear term decays by exactly the
integrating factor, a Taylor-Green vortex keeps its analytic viscous decay to the order
of its amplitude squared, and every step leaves the field divergence-free.

Follows, element by element and in their evaluation order:
  ADV_FLUID        adv_fluid.f90:47-187
  NONLINEAR_TERMS  nonlinear_terms.f90:81-160
  PROJ_DIVFREE     proj_divfree.f90:28-44
  wavenumbers      meshing.f90:96-140, filter meshing.f90:144-180, KFIRST/KLAST
                   init_run.f90:128-129, FACTOR main.f90:213
Arrays are [z][y][x] (x fastest), spectra [z][y][x/2+1] as numpy's rfftn over
axes (0, 1, 2) lays them out.  numpy's forward rfftn and backward irfftn(norm="forward")
are the unnormalised transforms P3DFFT's FTRAN/BTRAN are.
"""
from __future__ import annotations

import numpy as np

ZERO = 1.0e-33        # mod_dns_dim.f90:136
INFINITY = 1.0e33     # mod_dns_dim.f90:137


class Spectral:
    def __init__(self, nx, ny, nz, lx, visc, dtime, aliascontrol=2, rtrunc=8.0 / 9.0):
        self.shape = (nz, ny, nx)
        self.visc, self.dtime = visc, dtime
        ppi = 4.0 * np.arctan(1.0)
        self.ppi = ppi
        kfirst = 2.0 * ppi / lx
        self.klast = ppi / (lx / nx)
        self.factor = 1.0 / float(nx * ny * nz)
        kx = np.arange(nx // 2 + 1) * kfirst
        j = np.arange(ny)
        ky = np.where(j + 1 <= ny // 2 + 1, j, j - ny) * kfirst
        k = np.arange(nz)
        kz = np.where(k + 1 <= nz // 2 + 1, k, k - nz) * kfirst
        self.kx = kx[None, None, :]
        self.ky = ky[None, :, None]
        self.kz = kz[:, None, None]
        k2scl = (self.kx / self.klast) ** 2 + (self.ky / self.klast) ** 2 + (self.kz / self.klast) ** 2
        filt = np.ones_like(k2scl)
        if aliascontrol == 1:
            filt[k2scl > rtrunc * rtrunc] = 0.0
        elif aliascontrol == 2:
            band = (k2scl > rtrunc * rtrunc) & (k2scl <= 1.0)
            c = np.cos((ppi / 2.0) * (np.sqrt(k2scl) - rtrunc) / (1.0 - rtrunc))
            c2 = c * c
            filt = np.where(band, c2 * c2, filt)
            filt = np.where(k2scl > 1.0, 0.0, filt)
        self.filter = filt

    def fwd(self, a):
        return np.fft.rfftn(a, axes=(0, 1, 2))

    def bwd(self, a):
        return np.fft.irfftn(a, s=self.shape, axes=(0, 1, 2), norm="forward")

    def vorticity_hat(self, uh, vh, wh):
        """i k x û (nonlinear_terms.f90:81-92)."""
        def ik(a, k):
            return (-a.imag * k) + 1j * (a.real * k)
        ox = ik(wh, self.ky) - ik(vh, self.kz)
        oy = ik(uh, self.kz) - ik(wh, self.kx)
        oz = ik(vh, self.kx) - ik(uh, self.ky)
        return ox, oy, oz

    def nonlinear(self, u, v, w, uh, vh, wh):
        """NONLINEAR_TERMS added to RHS = cmplx(ZERO, ZERO)."""
        ox, oy, oz = self.vorticity_hat(uh, vh, wh)
        zx, zy, zz = self.bwd(ox), self.bwd(oy), self.bwd(oz)
        tx = v * zz - w * zy
        ty = w * zx - u * zz
        tz = u * zy - v * zx
        vx, vy, vz = (self.fwd(t) for t in (tx, ty, tz))
        vx, vy, vz = (_scale(a, self.factor) for a in (vx, vy, vz))
        kx, ky, kz = self.kx, self.ky, self.kz
        k2 = kx * kx + ky * ky + kz * kz
        k2 = np.where(k2 <= ZERO, INFINITY, k2)
        z = np.full(np.broadcast(kx, ky, kz).shape, ZERO + 1j * ZERO)
        ru = z + _scale(vx, (ky * ky + kz * kz) / k2) - _scale(vy, kx * ky / k2) - _scale(vz, kx * kz / k2)
        rv = z - _scale(vx, ky * kx / k2) + _scale(vy, (kx * kx + kz * kz) / k2) - _scale(vz, ky * kz / k2)
        rw = z - _scale(vx, kz * kx / k2) - _scale(vy, kz * ky / k2) + _scale(vz, (kx * kx + ky * ky) / k2)
        return ru, rv, rw

    def adv_fluid(self, u, v, w):
        """ADV_FLUID: one step; returns the new (u, v, w)."""
        dt = self.dtime
        uh, vh, wh = (_scale(self.fwd(a), self.factor) for a in (u, v, w))
        r = self.nonlinear(u, v, w, uh, vh, wh)
        kx, ky, kz = self.kx, self.ky, self.kz
        kappa2 = kx * kx + ky * ky + kz * kz
        ef = np.exp(-self.visc * kappa2 * dt)
        hats = [uh, vh, wh]
        np1 = [_scale(h + _scale(rc, dt / 2), ef) for h, rc in zip(hats, r)]
        hats = [_scale(h + _scale(rc, dt), ef) for h, rc in zip(hats, r)]
        u, v, w = (self.bwd(h) for h in hats)
        r = self.nonlinear(u, v, w, *hats)
        U, V, W = (a + _scale(rc, dt / 2) for a, rc in zip(np1, r))
        k2 = np.where(kappa2 <= ZERO, INFINITY, kappa2)
        divc = _scale(U, kx) + _scale(V, ky) + _scale(W, kz)
        U = U - _scale(divc, kx / k2)
        V = V - _scale(divc, ky / k2)
        W = W - _scale(divc, kz / k2)
        U, V, W = (_scale(a, self.filter) for a in (U, V, W))
        return self.bwd(U), self.bwd(V), self.bwd(W)

    def vorticity(self, u, v, w):
        uh, vh, wh = (_scale(self.fwd(a), self.factor) for a in (u, v, w))
        return tuple(self.bwd(o) for o in self.vorticity_hat(uh, vh, wh))

    def divergence_hat(self, u, v, w):
        uh, vh, wh = (self.fwd(a) for a in (u, v, w))
        return _scale(uh, self.kx) + _scale(vh, self.ky) + _scale(wh, self.kz)


def _scale(a, r):
    """complex times real, part by part"""
    return (a.real * r) + 1j * (a.imag * r)
