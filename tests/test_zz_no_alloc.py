"""gp_ellipsoid_contact_detection_batch_noalloc against gp_ellipsoid_contact_detection_batch.

The no-allocation entry point stages its work through one static device array that
every call shares; two calls in a row, the second smaller than the first and on other
pairs, check that it gives the context-based entry point's results each time and that
nothing of the first call leaks into the second.  The file is named so that pytest
collects it last, and it must pass alone in a fresh process as well."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gazpart_b200 import _lib, api, config
from _cases import REL_TOL

pytestmark = pytest.mark.gpu

MAX_PAIRS = 32768  # GP_NOALLOC_MAX_PAIRS in include/gazpart_gpu.h
EBADARG = 9        # GP_EBADARG


def _pairs(n: int, seed: int):
    """Pairs of ellipsoids placed from deep overlap to a clear gap, as the collision loop meets them."""
    rng = np.random.default_rng(seed)
    shapes = np.empty((n, 4))
    shapes[:, 0] = rng.uniform(0.004, 0.02, n)
    shapes[:, 1] = rng.uniform(0.3, 4.0, n)
    shapes[:, 2] = rng.uniform(0.004, 0.02, n)
    shapes[:, 3] = rng.uniform(0.3, 4.0, n)
    q = rng.normal(size=(n, 8))
    q[:, :4] /= np.linalg.norm(q[:, :4], axis=1, keepdims=True)
    q[:, 4:] /= np.linalg.norm(q[:, 4:], axis=1, keepdims=True)
    b1 = rng.uniform(0.0, 1.0, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    reach = (np.maximum(shapes[:, 0], shapes[:, 0] / shapes[:, 1])
             + np.maximum(shapes[:, 2], shapes[:, 2] / shapes[:, 3]))
    b2 = b1 + d * (reach * rng.uniform(0.2, 1.1, n))[:, None]
    return shapes, np.hstack([b1, b2]), q


def _noalloc(shapes, centres, quats):
    n = shapes.shape[0]
    flag = np.full(n, -7, dtype=np.int32)
    e1, e2, cn = (np.full((n, 3), np.nan) for _ in range(3))
    arrs = [np.ascontiguousarray(t) for t in (shapes, centres, quats)] + [flag, e1, e2, cn]
    rc = _lib.lib().gp_ellipsoid_contact_detection_batch_noalloc(
        n, *[C.c_void_p(t.ctypes.data) for t in arrs], 0, None)
    return rc, flag, e1, e2, cn


def _close(a, b):
    scale = np.maximum(np.abs(b), 1e-300)
    return bool(np.all(np.abs(a - b) <= REL_TOL * scale))


def test_noalloc_matches_context_entry_point_on_two_calls():
    with api.Context(config.Setup(nx=32, ny=32, nz=32), "fp64") as ctx:
        for n, seed in ((5000, 11), (1800, 12)):
            shapes, centres, quats = _pairs(n, seed)
            ref_flag, ref_e1, ref_e2, ref_cn = ctx.ellipsoid_contact_detection(shapes, centres, quats)
            rc, flag, e1, e2, cn = _noalloc(shapes, centres, quats)
            assert rc == 0
            assert np.array_equal(flag, ref_flag)
            assert 0 < int(flag.sum()) < n          # both outcomes are exercised
            for got, ref in ((e1, ref_e1), (e2, ref_e2), (cn, ref_cn)):
                assert _close(got, ref)


def test_noalloc_rejects_more_than_the_maximum():
    n = MAX_PAIRS + 1
    shapes = np.ones((n, 4))
    centres = np.zeros((n, 6))
    quats = np.zeros((n, 8))
    rc, flag, *_ = _noalloc(shapes, centres, quats)
    assert rc == EBADARG
    assert np.all(flag == -7)                       # nothing was written
