"""gp_ellipsoid_contact_detection_batch_noalloc against gp_ellipsoid_contact_detection_batch.

The no-allocation entry point serves callers that cannot allocate device memory (a
particle pool that already fills HBM, a real-time loop that cannot take cudaFree's
device synchronisation).  It stages its work through one static device array that every
call shares.  Two calls in a row, the second smaller than the first and on other pairs,
check that it gives the context-based entry point's results bit for bit each time (both
run the same contact solve without FMA contraction) and the oracle's, and that nothing
of the first call leaks into the second.  A third check runs it on device arrays and a
non-default stream.  The file is named so that pytest collects it last, and it must
pass alone in a fresh process as well."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import pyoracle as po
from gazpart_b200 import _lib, api, config

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


def _oracle(shapes, centres, quats, count):
    """The oracle's contact detection on the first `count` pairs."""
    out = []
    for i in range(count):
        s, c, q = shapes[i], centres[i], quats[i]
        r = po.contact_detection(s[0], s[1], s[2], s[3], c[:3], q[:4], c[3:], q[4:])
        out.append(r)
    return out


def _same(a, b):
    """Bit for bit, NaN where the other is NaN."""
    return bool(np.all((a == b) | (np.isnan(a) & np.isnan(b))))


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
                assert _same(got, ref)
            # and the oracle's solve, on a sample of the pairs
            for i, r in enumerate(_oracle(shapes, centres, quats, 400)):
                assert flag[i] == r["flag"], i
                for got, key in ((e1, "ept1"), (e2, "ept2"), (cn, "cnormal")):
                    assert _same(got[i], r[key]), (i, key)


def test_noalloc_device_arrays_on_a_side_stream():
    import torch
    shapes, centres, quats = _pairs(3000, 13)
    with api.Context(config.Setup(nx=32, ny=32, nz=32), "fp64") as ctx:
        ref_flag, ref_e1, ref_e2, ref_cn = ctx.ellipsoid_contact_detection(shapes, centres, quats)
    dev = torch.device("cuda", torch.cuda.current_device())
    ins = [torch.from_numpy(np.ascontiguousarray(t)).to(dev) for t in (shapes, centres, quats)]
    flag = torch.full((3000,), -7, dtype=torch.int32, device=dev)
    outs = [torch.full((3000, 3), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        rc = _lib.lib().gp_ellipsoid_contact_detection_batch_noalloc(
            3000, *[C.c_void_p(t.data_ptr()) for t in (*ins, flag, *outs)], 1, C.c_void_p(side.cuda_stream))
    assert rc == 0
    torch.cuda.current_stream().wait_stream(side)
    assert np.array_equal(flag.cpu().numpy(), ref_flag)
    for got, ref in zip(outs, (ref_e1, ref_e2, ref_cn)):
        assert _same(got.cpu().numpy(), ref)


def test_noalloc_refuses_a_stream_under_capture():
    """The call waits for its stream before returning, so on a stream being captured it
    returns GP_EBADARG with nothing enqueued and the caller's capture stays valid."""
    import torch
    shapes, centres, quats = _pairs(64, 14)
    x = torch.zeros(16, device="cuda")
    g = torch.cuda.CUDAGraph()
    flag = np.full(64, -7, dtype=np.int32)
    e1, e2, cn = (np.full((64, 3), np.nan) for _ in range(3))
    arrs = [np.ascontiguousarray(t) for t in (shapes, centres, quats)] + [flag, e1, e2, cn]
    with torch.cuda.graph(g):
        x.add_(1.0)
        rc = _lib.lib().gp_ellipsoid_contact_detection_batch_noalloc(
            64, *[C.c_void_p(t.ctypes.data) for t in arrs], 0,
            C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == EBADARG
    assert np.all(flag == -7)
    g.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0


def test_noalloc_rejects_more_than_the_maximum():
    n = MAX_PAIRS + 1
    shapes = np.ones((n, 4))
    centres = np.zeros((n, 6))
    quats = np.zeros((n, 8))
    rc, flag, *_ = _noalloc(shapes, centres, quats)
    assert rc == EBADARG
    assert np.all(flag == -7)                       # nothing was written
