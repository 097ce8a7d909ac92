"""Host-side logic that needs no GPU: the C ABI library's exports, the launch-choice
mapping of the Python mirror, the workload conventions, the field generator, the
particle initialiser and the replica timing reduction across ranks (gloo, two
processes)."""
from __future__ import annotations

import ctypes as C
import math
import os
import socket

import numpy as np
import pytest
import torch

from gazpart_b200 import _lib, config, field, particles


def test_library_exports_every_declared_symbol():
    names = _lib.exported_symbols()
    assert len(names) >= 25
    L = C.CDLL(_lib.LIB_PATH)
    for n in names:
        assert hasattr(L, n), n
    # the ctypes table binds exactly the declared entry points
    assert sorted(_lib.SIGNATURES) == names


def test_tuning_entry_points_refuse_bad_arguments():
    """The launch-tuning entry points check their arguments before they touch a device:
    a null context or output pointer, or an out-of-range choice, is GP_EBADARG."""
    L = _lib.lib()
    ebadarg = 9
    v = C.c_int32()
    assert L.gp_set_contact_order(None, 1) == ebadarg
    assert L.gp_get_contact_order(None, C.byref(v)) == ebadarg
    assert L.gp_set_gather_staging(None, 1) == ebadarg
    assert L.gp_get_gather_staging(None, C.byref(v)) == ebadarg
    assert L.gp_set_contact_tail(None, 4) == ebadarg


def test_params_struct_matches_header_layout():
    # gp_params: 3 int32, 11 doubles, 6 int32, 1 int64 with natural alignment
    assert C.sizeof(_lib.GPParams) == 3 * 4 + 4 + 11 * 8 + 6 * 4 + 8
    assert _lib.GPParams.max_particles.offset % 8 == 0


def test_workload_conventions():
    w = config.C1
    s = w.setup()
    t = config.integral_time()
    assert abs(t - math.sqrt(2 * math.pi) / 4) < 1e-15
    st = particles.draw(w.spec, s)
    assert np.all(st["rhop"] == 1000.0)
    deq = (2 * st["emaj"]) / st["apr"] ** (2 / 3)
    tau = (st["rhop"] / s.rhof) * deq ** 2 / (18 * s.visc)
    assert np.allclose(tau / t, 1.0)          # St = 1
    c3 = config.C3.spec
    small = config.ParticleSpec(**{**c3.__dict__, "n": 20000})
    st3 = particles.draw(small, config.C3.setup())
    deq3 = (2 * st3["emaj"]) / st3["apr"] ** (2 / 3)
    st_num = (st3["rhop"] / 1.0) * deq3 ** 2 / (18 * config.C3.setup().visc) / t
    assert st_num.min() >= 0.1 - 1e-9 and st_num.max() <= 10 + 1e-9
    assert (st3["apr"] < 1).any() and (st3["apr"] > 1).any()


def test_particles_drawn_inside_and_unit_quaternions():
    s = config.Setup(nx=32, ny=32, nz=32)
    spec = config.ParticleSpec(n=5000, ar_range=(0.2, 5.0), b=0.01, st=1.0, seed=3)
    st = particles.draw(spec, s)
    r = np.maximum(st["emaj"], st["emaj"] / st["apr"])
    for k, L in (("x", s.lx), ("y", s.ly), ("z", s.lz)):
        assert np.all(st[k] >= r) and np.all(st[k] <= L - r)
    qn = st["qa"] ** 2 + st["qb"] ** 2 + st["qc"] ** 2 + st["qd"] ** 2
    assert np.allclose(qn, 1.0)
    assert np.allclose(st["ipyy"], st["ipzz"])
    again = particles.draw(spec, s)
    assert all(np.array_equal(st[k], again[k]) for k in st)


def test_field_is_solenoidal_with_the_target_energy():
    n = 32
    f = field.generate(n, seed=0, device="cpu")
    e = 0.5 * sum(float((f[k] ** 2).mean()) for k in ("u", "v", "w"))
    assert abs(e - 1.5) < 1e-12
    period = n * (2 * math.pi / (n - 1))
    k = torch.fft.fftfreq(n, d=period / n, dtype=torch.float64) * 2 * math.pi
    kz, ky, kx = k.view(n, 1, 1), k.view(1, n, 1), k.view(1, 1, n)
    div = torch.fft.ifftn(1j * (kx * torch.fft.fftn(f["u"]) + ky * torch.fft.fftn(f["v"]) + kz * torch.fft.fftn(f["w"]))).real
    assert float(div.abs().max()) < 1e-10
    g = field.generate(n, seed=0, device="cpu")
    assert torch.equal(g["vortz"], f["vortz"])


def test_reference_layout_ghosts():
    rng = np.random.default_rng(0)
    a = torch.from_numpy(rng.normal(size=(5, 6, 7)))
    per = field.reference_layout(a, "periodic")
    zer = field.reference_layout(a, "zero")
    assert per.shape == (9, 10, 7)
    # J = 0 ghost plane (index 1) holds interior J = NY (index 5 of the interior)
    assert torch.equal(per[2:7, 1, :], a[:, 5, :])
    assert torch.equal(per[0, 2:8, :], a[3, :, :])
    assert torch.equal(zer[2:7, 2:8, :], a) and float(zer[0].abs().sum()) == 0.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    from bench import reduce_max_ms
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local = [12.5, 20.0][rank]
    out[rank] = reduce_max_ms(local, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_reduction_two_ranks():
    """bench.py --gpus N runs one replica per rank; the job time is the max over ranks."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == 20.0 and out[1] == 20.0


def test_batched_workload_instances():
    w = config.C4
    assert len(w.instances) == 64
    n = np.array([s.n for s in w.instances])
    assert n.min() >= 1000 and n.max() <= 2_000_000
    assert abs(n.sum() - 1.7e7) < 1e5                    # the stated total
    st = np.array([s.st for s in w.instances])
    ar = np.array([s.ar for s in w.instances])
    assert st.min() >= 0.1 and st.max() <= 10 and ar.min() >= 0.2 and ar.max() <= 5
    assert len({s.seed for s in w.instances}) == 64
    one = particles.draw(config.ParticleSpec(**{**w.instances[0].__dict__, "n": 500}), w.setup())
    deq = 2 * one["emaj"] / one["apr"] ** (2 / 3)
    st_num = one["rhop"] * deq ** 2 / (18 * w.setup().visc) / config.integral_time()
    assert np.allclose(st_num, w.instances[0].st)      # density follows the instance's Stokes number


def _shard_rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    counts = [s.n for s in config.C4.instances]
    mine = config.shard_instances(counts, world)[rank]
    n = torch.tensor([sum(counts[i] for i in mine)], dtype=torch.int64)
    dist.all_reduce(n)                                  # as bench.py sums the shares
    out[rank] = (mine, int(n.item()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_batched_classes_shard_over_ranks(world):
    """bench.py --gpus N splits the 64 classes of the 256^3 batched workload over the ranks: every class on one rank,
    the particle total summed across ranks equals the workload's, the shares balanced."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    counts = [s.n for s in config.C4.instances]
    shares = [out[r][0] for r in range(world)]
    assert sorted(i for sh in shares for i in sh) == list(range(64))
    assert all(out[r][1] == sum(counts) for r in range(world))
    loads = [sum(counts[i] for i in sh) for sh in shares]
    assert max(loads) - min(loads) <= max(counts)


def test_serving_stream_and_concurrency_count():
    from gazpart_b200 import serving
    w = config.C5
    jobs = w.jobs(50.0, seed=3)
    t = np.array([j[0] for j in jobs])
    assert np.all(np.diff(t) > 0) and t[-1] <= 50.0
    assert abs(len(jobs) / 50.0 - w.rate_per_s) < 3.0    # Poisson at 20/s
    steps = np.array([j[3] for j in jobs])
    n = np.array([j[2].n for j in jobs])
    assert steps.min() >= 100 and steps.max() <= 2000
    assert n.min() >= 1000 and n.max() <= 4_000_000
    assert set(j[1] for j in jobs) == set(range(len(w.fields)))
    fake = [serving.Job(state={"x": np.zeros(1)}, steps=1, admitted_s=a, done_s=d)
            for a, d in ((0.0, 2.0), (1.0, 3.0), (2.5, 4.0), (5.0, 6.0))]
    assert serving.max_concurrent(fake) == 2


class _FakeLaunchLib:
    """Stands in for the library's launch entry points: records what gp_set_launch
    receives and answers gp_autotune with a fixed choice."""

    def __init__(self, choice):
        self.choice, self.seen = choice, None

    def gp_set_launch(self, h, g):
        self.seen = [g[k] for k in range(len(_lib.TUNABLES) + 1)]
        return 0

    def gp_autotune(self, h, g):
        for k, v in enumerate([148, 296, 592, 1184, self.choice]):
            g[k] = v
        return 0

    def gp_set_contact_tail(self, h, b):
        return 0

    def gp_get_contact_tail(self, h, b):
        return 0

    def gp_set_gather_staging(self, h, m):
        self.staging = m
        return 0

    def gp_get_gather_staging(self, h, m):
        return 0


@pytest.mark.parametrize("choice", [0, 1, 2])
def test_launch_choices_map_to_the_abi(monkeypatch, choice):
    """gp_autotune's last value (0 no overlap, 1 gather overlapped, 2 gather and
    speculative integrate) round-trips through autotune() and set_launch()."""
    from gazpart_b200 import api
    fake = _FakeLaunchLib(choice)
    monkeypatch.setattr(_lib, "lib", lambda: fake)
    ctx = object.__new__(api.Context)
    ctx._h = None
    got = ctx.autotune()
    assert got["overlap_gather"] == (choice != 0)
    assert got["speculative_integrate"] == (choice == 2)
    ctx.set_launch(got)
    assert fake.seen == [148, 296, 592, 1184, choice]
    # the speculative integrate implies the overlap
    ctx.set_launch({"gather": 148, "integrate": 148, "bin": 148, "search": 148, "speculative_integrate": True})
    assert fake.seen[-1] == 2


def test_volume_fraction_known_answers():
    """bench.volume_fraction: a sphere and a prolate and an oblate spheroid (semi-axes
    EMAJ along the axis, EMAJ/APR across) in a unit box, and a list of classes."""
    import bench
    s = config.Setup(nx=8, ny=8, nz=8, lx=1.0, ly=1.0, lz=1.0)
    one = {"emaj": np.array([0.1]), "apr": np.array([1.0])}
    assert abs(bench.volume_fraction(one, s) - 4.0 / 3.0 * math.pi * 1e-3) < 1e-15
    pro = {"emaj": np.array([0.2]), "apr": np.array([2.0])}       # semi-axes 0.2, 0.1, 0.1
    obl = {"emaj": np.array([0.05]), "apr": np.array([0.5])}      # semi-axes 0.05, 0.1, 0.1
    v = 4.0 / 3.0 * math.pi * (0.2 * 0.01 + 0.05 * 0.01)
    assert abs(bench.volume_fraction([pro, obl], s) - v) < 1e-15
