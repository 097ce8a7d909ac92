"""B200 implementation of GAZPART's frozen-flow ellipsoidal-particle step.

The compute path is the CUDA library ``libgazpart_b200.so`` behind the C ABI in
``include/gazpart_gpu.h``; :mod:`gazpart_b200.api` mirrors the reference routines on
top of it, :mod:`gazpart_b200.field` and :mod:`gazpart_b200.particles` build the
seeded synthetic workloads of :mod:`gazpart_b200.config`.
"""
from . import config  # noqa: F401

__all__ = ["config"]
