"""Workload definitions for the frozen-flow ellipsoidal-particle step.

The reference reads its physical setup from ``param.in`` through ``READPARAM``
(``readparam.f90:8-277``) into module variables (``mod_param_phys.f90:14-113``).
Here one :class:`Setup` carries the values that the hot path reads
(``VISC``, ``RHOF``, ``DTIME``, ``GRAVITY``, ``ECP``/``MUP``, ``ECW``/``MUW``, mesh),
and one :class:`ParticleSpec` describes how a seeded ensemble of spheroids is drawn.

Conventions this module fixes (the reference has no Stokes-number parameter):

* fluid density ``RHOF = 1``; box ``L = 2*pi``; mesh spacing ``DX = L/(N-1)``
  (``meshing.f90:43-45``);
* particle relaxation time ``tau_p = (rho_p/rho_f) d_eq^2 / (18 nu)`` with the
  volume-equivalent diameter ``d_eq = 2 a / APR^(2/3)`` (``fluid_force_ellipsoid.f90:70``);
* Stokes number ``St = tau_p / T_int`` with the integral time of the synthetic
  spectrum ``T_int = L_int/u' = sqrt(2 pi)/(k0 u')``;
* the viscosity is fixed per workload so that the reference particle (median shape,
  geometric-mean Stokes number) has the nominal density ratio (1000); every particle's
  density is then set from its own Stokes number: ``rho_p = St 18 nu T_int / d_eq^2``.
* prolate spheroids (AR >= 1) have the symmetry semi-axis ``EMAJ = AR*b``; oblate ones
  (AR < 1) have ``EMAJ = b`` and equatorial semi-axes ``b/AR`` (the reference's
  ``ELL_B = ELL_A/APR``, ``calculate_ellipsoid_matrix.f90:33-35``).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

TWO_PI = 2.0 * math.pi


def integral_time(k0: float = 4.0, uprime: float = 1.0) -> float:
    """Integral time scale of E(k)=16 sqrt(2/pi) u'^2 k^4/k0^5 exp(-2k^2/k0^2)."""
    return math.sqrt(2.0 * math.pi) / (k0 * uprime)


@dataclasses.dataclass
class Setup:
    """Per-ensemble mesh and physics (the reference's module variables)."""
    nx: int
    ny: int
    nz: int
    lx: float = TWO_PI
    ly: float = TWO_PI
    lz: float = TWO_PI
    visc: float = 1.0e-2
    rhof: float = 1.0
    dtime: float = 1.0e-3
    gravity: float = 0.0
    ecp: float = 1.0
    mup: float = 0.0
    ecw: float = 1.0
    muw: float = 0.0
    periodicity: bool = True
    wall_boundary: bool = False
    frozen_flow: int = 2          # FROZEN_FLOW: 3 = channel (walls at x = 0, L; y and z wrap)

    @property
    def dx(self) -> float:
        return self.lx / float(self.nx - 1)

    @property
    def dy(self) -> float:
        return self.ly / float(self.ny - 1)

    @property
    def dz(self) -> float:
        return self.lz / float(self.nz - 1)

    @property
    def ppi(self) -> float:
        return 4.0 * math.atan(1.0)


@dataclasses.dataclass
class ParticleSpec:
    """How an ensemble's particles are drawn (the benchmark workload definitions)."""
    n: int
    # aspect ratio: fixed value, or log-uniform range (lo, hi)
    ar: Optional[float] = None
    ar_range: Optional[Tuple[float, float]] = None
    # minor semi-axis b: fixed, or log-normal (mu = ln median, sigma)
    b: Optional[float] = None
    b_lognormal: Optional[Tuple[float, float]] = None
    # Stokes number: fixed, uniform range, or log-uniform range
    st: Optional[float] = None
    st_uniform: Optional[Tuple[float, float]] = None
    st_loguniform: Optional[Tuple[float, float]] = None
    density_ratio: float = 1000.0
    seed: int = 1
    # distance kept between the particles and the x = 0 and x = L planes at t = 0 (at
    # least the particle's own largest semi-axis)
    x_margin: float = 0.0
    # monodisperse ensembles take exactly the nominal density ratio unless this is set,
    # in which case the density follows the Stokes number as for polydisperse ones
    density_from_st: bool = False

    def reference_shape(self) -> Tuple[float, float]:
        """(AR, b) of the median particle, used to fix the viscosity."""
        if self.ar is not None:
            ar = self.ar
        else:
            lo, hi = self.ar_range
            ar = math.sqrt(lo * hi)
        if self.b is not None:
            b = self.b
        else:
            b = math.exp(self.b_lognormal[0])
        return ar, b

    def reference_st(self) -> float:
        if self.st is not None:
            return self.st
        if self.st_uniform is not None:
            lo, hi = self.st_uniform
            return math.sqrt(lo * hi)
        lo, hi = self.st_loguniform
        return math.sqrt(lo * hi)


def shape_emaj_apr(ar: float, b: float) -> Tuple[float, float]:
    """(EMAJ, APR) of a spheroid with aspect ratio ``ar`` and minor semi-axis ``b``."""
    if ar >= 1.0:
        return ar * b, ar
    return b, ar


def d_equiv(emaj: float, apr: float) -> float:
    """Volume-equivalent diameter, fluid_force_ellipsoid.f90:70."""
    return (2.0 * emaj) / (apr ** (2.0 / 3.0))


def viscosity_for(spec: ParticleSpec, t_int: float) -> float:
    """Viscosity that gives the median particle the nominal density ratio."""
    ar, b = spec.reference_shape()
    emaj, apr = shape_emaj_apr(ar, b)
    d = d_equiv(emaj, apr)
    return spec.density_ratio * d * d / (18.0 * spec.reference_st() * t_int)


@dataclasses.dataclass
class Workload:
    name: str
    grid: int
    field_dtype: str          # "f64" or "f32"
    spec: ParticleSpec
    dtime: float
    steps: int
    field_seed: int = 0
    components: int = 6       # 6 = velocity + vorticity; 12 = velocity + 9 gradients

    def setup(self) -> Setup:
        t = integral_time()
        return Setup(nx=self.grid, ny=self.grid, nz=self.grid,
                     visc=viscosity_for(self.spec, t), dtime=self.dtime)


# The five workloads.  Particle counts and sizes are those of the benchmark
# definitions; unspecified time steps are 5e-4 (stable for St >= 0.1).
C1 = Workload("c1_64cube_n1e4_fp64", 64, "f64",
              ParticleSpec(n=10_000, ar=3.0, b=0.005, st=1.0, seed=1), 1.0e-3, 1000)
C2 = Workload("c2_256cube_n1e6_fp32field", 256, "f32",
              ParticleSpec(n=1_000_000, ar_range=(1.0, 5.0), b=0.002, st=0.5, seed=1), 5.0e-4, 500)
C3 = Workload("c3_512cube_n16777216_fp32field", 512, "f32",
              ParticleSpec(n=16_777_216, ar_range=(0.2, 5.0), b_lognormal=(math.log(1e-3), 0.3),
                           st_uniform=(0.1, 10.0), seed=1), 5.0e-4, 200)



@dataclasses.dataclass
class BatchedWorkload:
    """Independent ensembles (classes) on one shared field, stepped together."""
    name: str
    grid: int
    field_dtype: str
    instances: Tuple[ParticleSpec, ...]
    dtime: float
    steps: int
    field_seed: int = 0

    @property
    def spec(self) -> ParticleSpec:
        """The reference instance that fixes the shared viscosity."""
        return self.instances[0]

    def setup(self) -> Setup:
        return Setup(nx=self.grid, ny=self.grid, nz=self.grid,
                     visc=viscosity_for(_C4_REFERENCE, integral_time()), dtime=self.dtime)


def c4_instances(count: int = 64, seed: int = 193) -> Tuple[ParticleSpec, ...]:
    """64 instances: N log-uniform in [1e3, 2e6], one Stokes number log-uniform in
    [0.1, 10] and one aspect ratio log-uniform in [0.2, 5] per instance, minor semi-axis
    0.002 (the 256^3 field's particle size), each with its own seed.  The draw's seed is
    the one of 0..199 whose total comes closest to the stated sum N ~ 1.7e7
    (17,031,259 particles)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    n = np.exp(rng.uniform(math.log(1e3), math.log(2e6), count)).astype(int)
    st = np.exp(rng.uniform(math.log(0.1), math.log(10.0), count))
    ar = np.exp(rng.uniform(math.log(0.2), math.log(5.0), count))
    return tuple(ParticleSpec(n=int(n[i]), ar=float(ar[i]), b=0.002, st=float(st[i]), seed=1000 + i,
                              density_from_st=True) for i in range(count))


# the viscosity of the batched workload: a unit-aspect-ratio particle of b = 0.002 at
# St = 1 has the density ratio 1000
_C4_REFERENCE = ParticleSpec(n=1, ar=1.0, b=0.002, st=1.0)

C4 = BatchedWorkload("c4_256cube_64inst_fp32field", 256, "f32", c4_instances(), 5.0e-4, 300)


def shard_instances(counts: Sequence[int], world: int) -> List[List[int]]:
    """Instances of a batched workload split over `world` GPUs, each GPU one batched step
    over its share: largest first, each to the GPU with the fewest particles so far
    (ties to the lower rank).  Every instance lands on exactly one GPU; the shares are
    deterministic and differ by at most the largest instance."""
    loads = [0] * world
    shares: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(counts)), key=lambda k: (-counts[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        shares[r].append(i)
        loads[r] += counts[i]
    return [sorted(sh) for sh in shares]



@dataclasses.dataclass
class ServingWorkload:
    """A Poisson stream of tracking jobs on resident fields."""
    name: str
    fields: Tuple[Tuple[int, int], ...]     # (grid points per side, seed) of each resident field
    rate_per_s: float
    n_range: Tuple[float, float]            # log-uniform particle count
    steps_range: Tuple[int, int]            # uniform step count
    ar_range: Tuple[float, float]           # log-uniform aspect ratio, one per job
    st_range: Tuple[float, float]           # log-uniform Stokes number, one per job
    b: float
    dtime: float
    hbm_budget: float

    def setup(self, grid: int) -> Setup:
        return Setup(nx=grid, ny=grid, nz=grid, visc=viscosity_for(_C4_REFERENCE, integral_time()),
                     dtime=self.dtime)

    def jobs(self, window_s: float, seed: int = 5):
        """(arrival, field slot, spec, steps) of the jobs that arrive within window_s."""
        import numpy as np
        rng = np.random.default_rng(seed)
        t, out, j = 0.0, [], 0
        while True:
            t += rng.exponential(1.0 / self.rate_per_s)
            if t > window_s:
                return out
            n = int(np.exp(rng.uniform(math.log(self.n_range[0]), math.log(self.n_range[1]))))
            steps = int(rng.integers(self.steps_range[0], self.steps_range[1] + 1))
            ar = float(np.exp(rng.uniform(math.log(self.ar_range[0]), math.log(self.ar_range[1]))))
            st = float(np.exp(rng.uniform(math.log(self.st_range[0]), math.log(self.st_range[1]))))
            fid = int(rng.integers(0, len(self.fields)))
            out.append((t, fid, ParticleSpec(n=n, ar=ar, b=self.b, st=st, seed=1_000_000 + j,
                                             density_from_st=True), steps))
            j += 1


# Jobs at 20/s on eight resident FP32 fields (four 128^3, four 256^3), N log-uniform in
# [1e3, 4e6], steps uniform in [100, 2000], one aspect ratio and Stokes number per job,
# 150 GB of HBM for the jobs.  dt = 1e-4 keeps a 2000-step job clear of the x planes
# (see bench.x_margin_for).
C5 = ServingWorkload("c5_serving_8fields_20jobs_per_s", ((128, 0), (128, 1), (128, 2), (128, 3),
                                                        (256, 4), (256, 5), (256, 6), (256, 7)),
                     20.0, (1e3, 4e6), (100, 2000), (0.2, 5.0), (0.1, 10.0), 0.002, 1.0e-4, 150e9)

WORKLOADS = {w.name: w for w in (C1, C2, C3, C4)}
