"""Seeded solenoidal random-phase spectral field (synthetic frozen flow).

The reference initialises its frozen field in ``INITIATION_FROZEN_FLOW``
(``initiation_frozen_flow.f90:6-161``: zero field, a shear, or a channel profile read
from files that the reference does not ship).  The benchmark workloads instead use a
homogeneous isotropic random-phase field with the model spectrum

    E(k) = 16 sqrt(2/pi) u'^2 k^4 / k0^5 exp(-2 k^2 / k0^2),   k0 = 4, u' = 1,

and the vorticity computed spectrally.  This module builds that field; it is set-up
code, run once per ensemble with torch (FFT on the GPU when one is present).

Mesh semantics follow the reference: nodes sit at ``XMESH(i) = (i-1) DX`` with
``DX = L/(N-1)`` (``meshing.f90:43-55``) while the Lagrange stencil wraps with index
period ``N`` (``interp_lag3.f90:132-154``).  The field is therefore generated on an
``N``-point periodic grid of spacing ``DX`` (period ``N DX``), which makes the index
wrap consistent with the sampled field.

Random numbers come from a CPU ``torch.Generator`` seeded with ``seed`` and drawn
plane by plane, so the field is identical whatever device runs the FFTs.
"""
from __future__ import annotations

import math
from typing import Dict, Optional

import torch


def spectrum(k: torch.Tensor, k0: float = 4.0, uprime: float = 1.0) -> torch.Tensor:
    return 16.0 * math.sqrt(2.0 / math.pi) * uprime ** 2 * k ** 4 / k0 ** 5 * torch.exp(-2.0 * k ** 2 / k0 ** 2)


def _wavenumbers(n: int, length: float, device) -> torch.Tensor:
    return torch.fft.fftfreq(n, d=length / n, device=device, dtype=torch.float64) * (2.0 * math.pi)


def generate(n: int, lbox: float = 2.0 * math.pi, seed: int = 0, k0: float = 4.0,
             uprime: float = 1.0, device: Optional[str] = None,
             gradients: bool = False) -> Dict[str, torch.Tensor]:
    """Return the interior field as float64 tensors of shape (N, N, N) = [z][y][x].

    Keys: ``u, v, w, vortx, vorty, vortz`` and, with ``gradients``, ``dudx ..`` as
    ``grad[i][j] = d u_i / d x_j`` under keys ``g00 .. g22``.
    """
    if device is None:
        device = "cuda" if torch.cuda.is_available() else "cpu"
    dx = lbox / float(n - 1)
    period = n * dx
    kv = _wavenumbers(n, period, device)
    kz = kv.view(n, 1, 1)
    ky = kv.view(1, n, 1)
    kx = kv.view(1, 1, n)
    gen = torch.Generator(device="cpu")
    gen.manual_seed(int(seed))
    g = torch.empty((3, n, n, n), dtype=torch.complex128, device=device)
    for z in range(n):
        re = torch.randn((3, n, n), generator=gen, dtype=torch.float64)
        im = torch.randn((3, n, n), generator=gen, dtype=torch.float64)
        g[:, z] = torch.complex(re, im).to(device)
    k2 = kx * kx + ky * ky + kz * kz
    kmag = torch.sqrt(k2)
    # project onto the plane normal to k (solenoidal), then unit complex norm
    kdotg = kx * g[0] + ky * g[1] + kz * g[2]
    safe_k2 = torch.where(k2 > 0, k2, torch.ones_like(k2))
    g[0] -= kx * kdotg / safe_k2
    g[1] -= ky * kdotg / safe_k2
    g[2] -= kz * kdotg / safe_k2
    del kdotg
    gnorm = torch.sqrt((g.real ** 2 + g.imag ** 2).sum(0))
    dk = 2.0 * math.pi / period
    amp = torch.sqrt(2.0 * spectrum(kmag, k0, uprime) * dk ** 3 /
                     (4.0 * math.pi * torch.where(k2 > 0, k2, torch.ones_like(k2))))
    nyq = torch.zeros((n, n, n), dtype=torch.bool, device=device)
    if n % 2 == 0:
        h = n // 2
        nyq[h, :, :] = True
        nyq[:, h, :] = True
        nyq[:, :, h] = True
    scale = torch.where((k2 > 0) & (~nyq) & (gnorm > 0), amp / torch.where(gnorm > 0, gnorm, torch.ones_like(gnorm)),
                        torch.zeros_like(amp))
    del amp, gnorm, nyq
    g *= scale
    del scale
    vel = []
    for c in range(3):
        vel.append(torch.fft.ifftn(g[c]).real * float(n) ** 3)
    del g
    # fix the level exactly: (1/2)<|u|^2> = (3/2) u'^2
    e = 0.5 * sum((v * v).mean() for v in vel)
    fac = math.sqrt(1.5 * uprime ** 2 / float(e))
    vel = [v * fac for v in vel]
    out = {"u": vel[0], "v": vel[1], "w": vel[2]}
    # spectral derivatives of the (real) field
    kvec = (kx, ky, kz)
    hat = [torch.fft.fftn(v) for v in vel]
    def deriv(i: int, j: int) -> torch.Tensor:
        return torch.fft.ifftn(1j * kvec[j] * hat[i]).real
    out["vortx"] = deriv(2, 1) - deriv(1, 2)
    out["vorty"] = deriv(0, 2) - deriv(2, 0)
    out["vortz"] = deriv(1, 0) - deriv(0, 1)
    if gradients:
        for i in range(3):
            for j in range(3):
                out[f"g{i}{j}"] = deriv(i, j)
    return out


COMPONENTS_6 = ("u", "v", "w", "vortx", "vorty", "vortz")


def reference_layout(interior: torch.Tensor, ghost: str) -> torch.Tensor:
    """Embed an interior (NZ, NY, NX) array into the reference's ghosted layout.

    Returns shape (NZ+4, NY+4, NX) -- Fortran ``(NX, NY+4, NZ+4)`` with x fastest
    (``allocate_arrays.f90:93-118``, ``NGHTCELL = 2``).  ``ghost`` is ``"periodic"``
    (what ``FLUIDCOMM`` produces on one rank, ``MPI_structures.f90:84-132``) or
    ``"zero"`` (the vorticity arrays, whose ghosts are never exchanged,
    ``main.f90:255-259``).
    """
    nz, ny, nx = interior.shape
    out = torch.zeros((nz + 4, ny + 4, nx), dtype=interior.dtype, device=interior.device)
    out[2:nz + 2, 2:ny + 2, :] = interior
    if ghost == "periodic":
        # y ghosts: J=-1,0 <- NY-1,NY ; J=NY+1,NY+2 <- 1,2   (planes of the full z range)
        out[2:nz + 2, 0:2, :] = interior[:, ny - 2:ny, :]
        out[2:nz + 2, ny + 2:ny + 4, :] = interior[:, 0:2, :]
        # z ghosts including y-ghost corners
        out[0:2, :, :] = out[nz:nz + 2, :, :]
        out[nz + 2:nz + 4, :, :] = out[2:4, :, :]
    elif ghost != "zero":
        raise ValueError(f"ghost must be 'periodic' or 'zero', not {ghost!r}")
    return out


# ---------------------------------------------------------------------------------
# Channel profile (FROZEN_FLOW = 3)
# ---------------------------------------------------------------------------------
CHANNEL_POINTS = 21   # N of initiation_frozen_flow.f90:80


def read_channel_profiles(ug_path: str, vorty_path: str):
    """The two profile files INITIATION_FROZEN_FLOW reads (initiation_frozen_flow.f90:
    82-93): 'Ug_mean.in', 21 records of (x, mean streamwise velocity), and
    'vorticity_y.txt', 21 records of the y vorticity, each read list-directed."""
    from .params import _ListReader
    ru = _ListReader(open(ug_path).read())
    rv = _ListReader(open(vorty_path).read())
    x_in, ug_in, vorty_in = [], [], []
    for _ in range(CHANNEL_POINTS):
        x, u = ru.read("rr")
        x_in.append(x)
        ug_in.append(u)
        vorty_in.append(rv.read("r")[0])
    return x_in, ug_in, vorty_in


def channel(setup, x_in, ug_in, vorty_in, frozen_interp) -> Dict[str, torch.Tensor]:
    """The frozen channel field of initiation_frozen_flow.f90:77-155 on the mesh
    XMESH(i) = (i-1) L/(N-1), interior arrays (NZ, NY, NX) = [z][y][x].

    The 21 profile values fill 21^3 tables constant in y and z; FROZEN_INTERP_LAG3
    samples them at the mesh diagonal (XMESH(i), YMESH(i), ZMESH(i)), i = 1..NX for the
    velocity and 1..NY for the vorticity.  Then U = V = 0, W(i,:,:) = WINT(i),
    VORTICITY_Y(:,j,:) = VORTY_INT(j) -- the vorticity profile lies along y, as the
    reference assigns it -- and the other vorticity components are 0.  The diagonal
    reads YMESH and ZMESH up to index NX and XMESH up to NY, so the reference needs
    NY, NZ >= NX and NX >= NY; other meshes are refused.

    frozen_interp(xain, yain, zain, uain, x, y, z) is FROZEN_INTERP_LAG3 with uain of
    shape (NZA, NYA, NXA): the device's (Context.frozen_interp_lag3) or the oracle's."""
    import numpy as np
    n = CHANNEL_POINTS
    nx, ny, nz = setup.nx, setup.ny, setup.nz
    if not (ny >= nx and nz >= nx and nx >= ny):
        raise ValueError("the channel profile needs NY = NX <= NZ (the reference's mesh-diagonal sampling)")
    x_in = np.asarray(x_in, dtype=np.float64)
    y_in = setup.ly / float(n - 1) * np.arange(n, dtype=np.float64)    # dy_frozen*(I-1)
    z_in = setup.lz / float(n - 1) * np.arange(n, dtype=np.float64)
    wtmp = np.broadcast_to(np.asarray(ug_in, dtype=np.float64)[None, None, :], (n, n, n)).copy()
    vtmp = np.broadcast_to(np.asarray(vorty_in, dtype=np.float64)[None, None, :], (n, n, n)).copy()
    xmesh = setup.dx * np.arange(nx, dtype=np.float64)
    ymesh = setup.dy * np.arange(ny, dtype=np.float64)
    zmesh = setup.dz * np.arange(nz, dtype=np.float64)
    wint = frozen_interp(x_in, y_in, z_in, wtmp, xmesh[:nx], ymesh[:nx], zmesh[:nx])
    vorty_int = frozen_interp(x_in, y_in, z_in, vtmp, xmesh[:ny], ymesh[:ny], zmesh[:ny])
    zero = torch.zeros((nz, ny, nx), dtype=torch.float64)
    w = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(wint[None, None, :], (nz, ny, nx))))
    vy = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(vorty_int[None, :, None], (nz, ny, nx))))
    return {"u": zero.clone(), "v": zero.clone(), "w": w, "vortx": zero.clone(), "vorty": vy, "vortz": zero.clone()}
