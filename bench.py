"""Benchmark of the frozen-flow ellipsoidal-particle step (particle-steps/s).

Default workload: 512^3 FP32 frozen field, 16,777,216 polydisperse spheroids
(AR log-uniform [0.2, 5], b log-normal(ln 1e-3, 0.3), St uniform [0.1, 10]),
dt = 5e-4, collisions on, mixed-precision form, one CUDA-graph step per iteration.

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]``

* ours: W untimed steps, then K steps timed with CUDA events on the library's stream
  (one captured graph of K steps with events around every phase), barrier and max over
  ranks; N>1 runs independent replicas (one ensemble per GPU, no collective in the step).
* reference: the CPU restatement of the reference algorithm (candidate pairs solved
  with Levenberg-Marquardt without a prefilter, as the reference does) timed on the
  host cores on a bounded sample with the workload's particle density and sizes.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3_512cube_n16777216_fp32field")
    ap.add_argument("--precision", default=None, choices=[None, "mixed", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 comparison run")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch grids")
    ap.add_argument("--no-io", action="store_true", help="skip the restart-file measurement")
    ap.add_argument("--no-stats", action="store_true", help="skip the statistics measurement")
    ap.add_argument("--no-dns", action="store_true", help="skip the live-fluid measurement")
    ap.add_argument("--no-forms", action="store_true", help="skip the batched and serving sub-benchmarks")
    ap.add_argument("--contact-tail", type=int, default=None,
                    help="evaluations after which a contact solve moves to the inlined-solver kernel (0: never)")
    ap.add_argument("--grids", default=None,
                    help="gather,integrate,bin,search,overlap[,contact_tail]: fixed launch choices instead of "
                         "autotuning (overlap 0: none, 1: gather, 2: gather and speculative integrate)")
    ap.add_argument("--serve-seconds", type=float, default=2.0, help="arrival window of the serving workload")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# workload construction
# ---------------------------------------------------------------------------
# steps the autotuner moves the particles before it restores them (gp_autotune): one-step
# graphs for each of the 4 launch grids at 5 sizes, 3 each; then eight-step graphs, 3 each,
# for up to 5 overlap choices (none; the gather at two grids; the gather and the
# speculative integrate at two grids)
AUTOTUNE_STEPS = 4 * 5 * 3 + 5 * 3 * 8


def volume_fraction(states, setup) -> float:
    """Solid volume fraction of the drawn particles: each spheroid has the semi-axis EMAJ
    along its axis and EMAJ / APR across it (calculate_ellipsoid_matrix.f90), so its
    volume is (4/3) pi EMAJ (EMAJ / APR)^2; the sum over the box volume."""
    import numpy as np
    sts = states if isinstance(states, list) else [states]
    v = sum(float(np.sum(4.0 / 3.0 * np.pi * s["emaj"] * (s["emaj"] / s["apr"]) ** 2)) for s in sts)
    return v / (setup.lx * setup.ly * setup.lz)


def x_margin_for(w, steps: int) -> float:
    """Distance from the x planes at which the run's particles start.

    The reference tests every particle against the planes x = 0 and x = L even in a
    periodic box (adv_particle_new.f90:331-336,555-560) and rebounds the ones that reach
    them.  At dt = 5e-4 the spin such a rebound gives a slender spheroid (about 7e3 rad/s
    about its axis) makes the explicit RK2 update of the angular velocity grow about
    five-fold per step until the drag coefficient is NaN and the run stops ('In Fluid
    force'); the FP64 path, which follows the reference bit for bit, stops on the same
    particle at the same step.  So the benchmark keeps every particle further from the
    x planes than a particle moving at 6 u' (beyond the fluid's largest velocity
    component) travels in the steps of the run."""
    return min(w.setup().lx / 4.0, 1.1 * 6.0 * w.dtime * steps)


def build_inputs(w, device, precision, steps: int = 0, rank: int = 0, world: int = 1):
    """Field and particles of a workload; a batched workload gives one state per class,
    and on several GPUs only this rank's share of the classes (config.shard_instances)."""
    import dataclasses
    import torch
    from gazpart_b200 import config, field, particles
    setup = w.setup()
    f = field.generate(w.grid, seed=w.field_seed, device=device)
    specs = w.instances if isinstance(w, config.BatchedWorkload) else (w.spec,)
    if isinstance(w, config.BatchedWorkload) and world > 1:
        share = config.shard_instances([sp.n for sp in specs], world)[rank]
        specs = tuple(specs[i] for i in share)
    m = x_margin_for(w, steps) if steps else 0.0
    states = [particles.draw(dataclasses.replace(sp, x_margin=m), setup) for sp in specs]
    return setup, f, states if isinstance(w, config.BatchedWorkload) else states[0]


def make_context(setup, f, st, precision, device):
    import torch
    from gazpart_b200 import api, particles
    ctx = api.Context(setup, precision)
    ctx.set_fields({k: f[k].contiguous() for k in api.FIELD_KEYS})
    states = st if isinstance(st, list) else [st]
    for one in states:
        # initial velocities: u = u_f(x), omega = 1/2 omega_f in the body frame
        xs = [torch.from_numpy(one[k]).to(device) for k in ("x", "y", "z")]
        g = [ctx.interp_lag3(c, *xs).cpu().numpy() for c in range(6)]
        one["u"], one["v"], one["w"] = g[0], g[1], g[2]
        particles.body_half_vorticity(one, g[3], g[4], g[5])
    if isinstance(st, list):
        ctx.upload_classes(states)
    else:
        ctx.upload(st)
    return ctx


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        finally:
            try:
                os.unlink(self.path)
            except OSError:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# measured peaks
# ---------------------------------------------------------------------------
def hbm_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def reduce_max_ms(ms: float, dist, device) -> float:
    """Job time of N replicas: the slowest rank's device time (max over ranks)."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_bytes_per_particle(components: int, field_bytes: int) -> int:
    """Algorithmic bytes of one particle in the stencil-gather kernel (k_gather):
    64 stencil points x C components x field word, the position read (24 B) and the C
    interpolated values written (8 B each, as the reference stores them).  No credit is
    taken for stencil reuse between particles; the reordering copy of the particle
    record that the kernel also performs is not algorithmic and is not counted."""
    return 64 * components * field_bytes + 24 + 8 * components


# DRAM bytes (read + write) per particle of one k_gather launch, from ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on the steady-state step; the file under
# profiles/ named in the value gives the command and the capture.  The gather's warps
# take consecutive runs of the cell order from one counter, so the figure does not
# depend on the gather's grid.
GATHER_TRAFFIC = {
    ("c3_512cube_n16777216_fp32field", "mixed"): (286.2, "profiles/k_gather_k_integrate_c3_dram.md"),
}


# ---------------------------------------------------------------------------
# CPU baseline: the restatement of the reference algorithm on the host cores
# ---------------------------------------------------------------------------
def cpu_sample(w, scale: int, max_emaj: float):
    """A periodic box of side L/scale with the workload's particle density and size
    distribution; the collision box edge is taken from the full workload's largest
    particle so each particle sees the same candidate count as in the full run."""
    import torch
    from gazpart_b200 import config, field, particles
    import pyoracle as po
    base = w.setup()
    n_s = max(8, w.grid // scale)
    L = base.lx / scale
    setup = config.Setup(nx=n_s, ny=n_s, nz=n_s, lx=L, ly=L, lz=L, visc=base.visc, dtime=base.dtime)
    spec = config.ParticleSpec(**{**w.spec.__dict__, "n": max(64, w.spec.n // scale ** 3), "seed": 77})
    f = field.generate(n_s, lbox=L, seed=1, device="cpu")
    refs = [field.reference_layout(f[k], "periodic" if k in ("u", "v", "w") else "zero").numpy().copy()
            for k in field.COMPONENTS_6]
    st = particles.draw(spec, setup)
    uf = [po.interp_lag3(setup, refs[c], st["x"], st["y"], st["z"]) for c in range(6)]
    st["u"], st["v"], st["w"] = uf[0].copy(), uf[1].copy(), uf[2].copy()
    particles.body_half_vorticity(st, uf[3], uf[4], uf[5])
    ens = po.Ensemble(setup, st)
    g = po.OrcBoxGrid()
    po.lib().orc_collision_initiation(po.C.byref(po.make_setup(setup)), po.C.c_double(max_emaj), po.C.byref(g))
    return ens, refs, g


def phase_note(tune) -> str:
    """What the multi-step graph's phase times cover under the launch choices in use."""
    if not tune or not tune.get("overlap_gather"):
        return "one stream: each phase alone"
    if tune.get("speculative_integrate"):
        return ("gather and integrate of step s+1 (particles in none of step s's candidate pairs) overlap the "
                "contact solves of step s on a second stream; 'integrate' times the pair members after the response")
    return "gather of step s+1 overlaps the contact solves of step s (two streams in the graph)"


def time_cpu(w, steps: int, threads: int, scale: int, max_emaj: float):
    ens, refs, g = cpu_sample(w, scale, max_emaj)
    t_adv = t_col = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        rc = ens.advance(refs, nthreads=threads)
        t1 = time.perf_counter()
        res = ens.collide(prefilter=False, nthreads=threads, grid=g)
        t2 = time.perf_counter()
        t_adv += t1 - t0
        t_col += t2 - t1
        if rc or res["rc"]:
            break
    per_step = (t_adv + t_col) / steps
    return {"value": ens.n / per_step, "n": ens.n, "steps": steps, "t_adv": t_adv / steps,
            "t_col": t_col / steps, "candidates_per_step": res["n_candidates"], "nbox": g.nbox}


def time_cpu_one_thread(w, scale: int, max_emaj: float, fraction: float = 0.01, seed: int = 3):
    """The same sample on one host thread, as the reference runs per MPI rank: the whole
    advance, and the collision phase timed on a random `fraction` of the step's candidate
    pairs (each evaluated as collision_interaction.f90:216-348 does, one Levenberg-Marquardt
    solve per pair) and scaled to all of them."""
    import pyoracle as po
    ens, refs, g = cpu_sample(w, scale, max_emaj)
    t0 = time.perf_counter()
    rc = ens.advance(refs, nthreads=1)
    t_adv = time.perf_counter() - t0
    if rc:
        raise RuntimeError(f"oracle advance failed ({rc})")
    ncon, con = ens.connectivity(g)
    a = ens.a
    xyz = [po.dptr(a[k]) for k in ("x", "y", "z")]
    ncand = po.lib().orc_detect_pairs(po.C.byref(g), po.iptr(ncon), po.iptr(con), po.C.c_int64(ens.n), *xyz,
                                      po.C.c_int64(0), None, None)
    home = np.zeros(ncand, dtype=np.int32)
    near = np.zeros(ncand, dtype=np.int32)
    po.lib().orc_detect_pairs(po.C.byref(g), po.iptr(ncon), po.iptr(con), po.C.c_int64(ens.n), *xyz,
                              po.C.c_int64(ncand), po.iptr(home), po.iptr(near))
    pick = np.random.default_rng(seed).choice(ncand, size=max(1, int(fraction * ncand)), replace=False)
    s, props, st = po.make_setup(ens.setup), ens.props(), ens.state()
    out = [np.zeros(3) for _ in range(5)]
    flag = po.C.c_int32()
    t0 = time.perf_counter()
    for e in pick:
        po.lib().orc_pair_eval(po.C.byref(s), po.C.byref(props), po.C.byref(st), po.C.c_int64(int(home[e])),
                               po.C.c_int64(int(near[e])), *[po.dptr(o) for o in out], po.C.byref(flag))
    t_pairs = time.perf_counter() - t0
    t_col = t_pairs * ncand / pick.size
    return {"value": ens.n / (t_adv + t_col), "n": ens.n, "t_adv": t_adv, "t_col": t_col,
            "candidates_per_step": int(ncand), "pairs_timed": int(pick.size)}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def reference_compilers() -> dict:
    """Where the reference's own Fortran toolchain is on this host (None: absent)."""
    import shutil
    return {t: shutil.which(t) for t in ("gfortran", "mpif90", "ifort", "ifx", "flang")}


def compare_mixed_fp64(w, device, steps: int, grids=None) -> dict:
    """The mixed form against the plain FP64 path on the full workload: both start from
    the same particles and take `steps` steps; every step the accepted pairs of the two
    are compared, and at the end the velocity error of the mixed form against the FP64
    path (which follows the oracle bit for bit up to libm) is reported, over every
    particle and over those that collided in neither run."""
    import torch
    setup, f, st = build_inputs(w, device, "mixed", steps)
    st64 = {k: np.array(v, copy=True) for k, v in st.items()}
    cm = make_context(setup, f, st, "mixed", device)
    cf = make_context(setup, {k: v for k, v in f.items()}, st64, "fp64", device)
    if grids:
        cm.set_launch({**grids, "overlap_gather": False, "speculative_integrate": False})
    n = cm.n
    collided = np.zeros(n, dtype=bool)
    flips, accepted, per_step = 0, 0, []
    for _ in range(steps):
        cm.step(1)
        cf.step(1)
        hm, nm = cm.collision_pairs()
        hf, nf = cf.collision_pairs()
        for h, nn in ((hm, nm), (hf, nf)):
            collided[h] = True
            collided[nn] = True
        a = set(zip(hm.tolist(), nm.tolist()))
        b = set(zip(hf.tolist(), nf.tolist()))
        flips += len(a ^ b)
        accepted += len(b)
        per_step.append(len(a ^ b))
    cm.raise_status("mixed comparison steps")
    cf.raise_status("fp64 comparison steps")
    gm, gf = cm.download(), cf.download()
    cm.close()
    cf.close()
    del cm, cf
    torch.cuda.empty_cache()
    du = np.sqrt(sum((gm[k] - gf[k]) ** 2 for k in ("u", "v", "w")))
    nu = np.sqrt(sum(gf[k] ** 2 for k in ("u", "v", "w")))
    err = du / (nu + 1e-30)
    free = err[~collided]
    dx = np.sqrt(sum((gm[k] - gf[k]) ** 2 for k in ("x", "y", "z")))
    return {"steps": steps, "particles": n, "velocity_rel_err": {
                "max_never_collided": float(free.max()), "p99_never_collided": float(np.quantile(free, 0.99)),
                "median_never_collided": float(np.median(free)), "max_all": float(err.max()),
                "p99_all": float(np.quantile(err, 0.99)), "median_all": float(np.median(err))},
            "position_abs_err_max": float(dx.max()),
            "never_collided": int((~collided).sum()),
            "pair_flips_total": flips, "pair_flips_per_step": per_step, "accepted_pairs_fp64": accepted,
            "target": "<= 1e-5 relative velocity error against the FP64 path"}


def time_batched(args, device) -> dict:
    """The batched workload (64 classes on one shared 256^3 field) in the same process
    after the single-ensemble run: autotuned grids, warm-up, one timed graph."""
    import torch
    from gazpart_b200 import config
    w = config.C4
    steps = max(5, args.steps // 2)
    run_steps = args.warmup + steps + AUTOTUNE_STEPS + 6
    setup, f, st = build_inputs(w, device, "mixed", run_steps)
    ctx = make_context(setup, f, st, "mixed", device)
    tune = None if args.no_autotune else ctx.autotune()
    ctx.step(args.warmup)
    ctx.sync()
    torch.cuda.synchronize()
    total_ms, phases, kps = ctx.step_timed(steps)
    ctx.raise_status("batched steps")
    n = ctx.n
    ctx.close()
    del ctx
    torch.cuda.empty_cache()
    return {"workload": w.name, "value": n * steps / (total_ms / 1e3), "unit": "particle-steps/s",
            "classes": len(st), "particles": n, "steps": steps, "ms_per_step": total_ms / steps,
            "phase_ms": phases, "kernels_per_step": kps, "launch_grids": tune}


def workload_max_emaj(w) -> float:
    from gazpart_b200 import particles
    st = particles.draw(w.spec, w.setup())
    return float(st["emaj"].max())


# ---------------------------------------------------------------------------
# serving: a Poisson job stream through gp_serve
# ---------------------------------------------------------------------------
def time_restart_io(ctx, n: int, state) -> dict:
    """The ensemble as a class restart file (save_particle.f90:116-180 layout): written
    straight from the device by gp_save_part_class and read back by gp_read_part_class,
    with a check that the file holds the state the context holds (state: the host copy
    of the current state, in particle order).  The file carries one table entry per
    class; the per-particle shapes of the synthetic workloads are not part of it."""
    import shutil
    from gazpart_b200 import restart
    tables = restart.default_tables(n, 1.0, 1.0, 1.0)
    d = tempfile.mkdtemp(prefix="gp_restart_")
    path = os.path.join(d, restart.part_file_name(1, 0))
    try:
        t0 = time.perf_counter()
        restart.save_class(ctx, 1, path, tables)
        t1 = time.perf_counter()
        cols, _ = restart.read_part_class(path)
        t2 = time.perf_counter()
        size = os.path.getsize(path)
        same = all(np.array_equal(cols[k], state[k]) for k in state)
        return {"file": restart.part_file_name(1, 0), "bytes": size, "particles": n,
                "save_s": t1 - t0, "save_gbs": size / (t1 - t0) / 1e9,
                "read_s": t2 - t1, "read_gbs": size / (t2 - t1) / 1e9, "matches_state": bool(same),
                "note": "save = D2H into pageable memory + write; read right after the write (page cache)"}
    except Exception as e:      # a full or read-only scratch disk leaves the step numbers valid
        return {"error": str(e)}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def time_stats(ctx) -> dict:
    """Statistics beside the step on the whole ensemble: STAT_PARTFLUID of class 1
    (one kernel over the pool, its 36 sums copied out; median of three calls, each
    synchronised) and the cost of the collision statistics in a step (four-step graphs
    with and without them, median of three each)."""
    import statistics as stt
    t = []
    for _ in range(3):
        t0 = time.perf_counter()
        m = ctx.stat_partfluid(1)
        t.append(time.perf_counter() - t0)
    out = {"partfluid_ms": 1e3 * stt.median(t), "partfluid_count": int(m[0, -1]),
           "partfluid_mean_rep": float(m[0, 0])}
    steps = {}
    for on in (False, True):
        ctx.enable_collision_stats(on)
        steps[on] = stt.median(ctx.step_timed(4)[0] for _ in range(3)) / 4
    cs, nsteps = ctx.collision_stats(1)
    ctx.enable_collision_stats(False)
    out.update({"step_ms": steps[False], "step_ms_with_collision_stats": steps[True],
                "collision_stats_steps": nsteps, "contacts_examined_per_step": float(cs[0, 0, 0]) / max(nsteps, 1),
                "collisions_per_step": float(cs[0, 0, 1]) / max(nsteps, 1)})
    return out


def time_live_fluid(ctx, setup, f) -> dict:
    """The live-fluid step (ADV_FLUID, gp_adv_fluid) on the workload's own mesh, started
    from its field, and the refresh of the context's field from it (gp_dns_couple):
    median of three synchronised calls each, after one untimed step."""
    import statistics as stt
    from gazpart_b200 import dns
    out = {"mesh": f"{setup.nx}x{setup.ny}x{setup.nz}", "ffts_per_step": 21}
    with dns.Fluid(setup) as fl:
        fl.set_velocity(f["u"], f["v"], f["w"])
        fl.adv_fluid(0)
        t = []
        for k in range(3):
            t0 = time.perf_counter()
            fl.adv_fluid(k + 1)
            t.append(time.perf_counter() - t0)
        c = []
        for _ in range(3):
            t0 = time.perf_counter()
            fl.couple(ctx)
            c.append(time.perf_counter() - t0)
    points = setup.nx * setup.ny * setup.nz
    out.update({"adv_fluid_ms": 1e3 * stt.median(t), "couple_ms": 1e3 * stt.median(c),
                "mesh_points_per_s": points / stt.median(t)})
    return out


def run_serving(args, rank: int, world: int, local: int, emit: bool = True):
    """Jobs arriving at 20/s for --serve-seconds, each on one of eight resident fields,
    admitted against the HBM budget and stepped together until all are done.  Prints the
    serving line (emit) or returns its fields."""
    import dataclasses
    import torch
    from gazpart_b200 import api, config, field, particles, serving
    w = config.C5
    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    stream = w.jobs(args.serve_seconds, seed=5 + rank)
    fields = [field.generate(n, seed=sd, device=device) for n, sd in w.fields]
    jobs = []
    for fid, (n, _) in enumerate(w.fields):
        mine = [(t, spec, steps) for t, f_, spec, steps in stream if f_ == fid]
        if not mine:
            continue
        setup = w.setup(n)
        with api.Context(setup, "mixed") as tmp:
            tmp.set_fields({k: fields[fid][k].contiguous() for k in api.FIELD_KEYS})
            for t, spec, steps in mine:
                # the largest job also carries the autotuner's trials before it leaves
                m = min(setup.lx / 4.0, 1.1 * 6.0 * w.dtime * max(steps, AUTOTUNE_STEPS + 6))
                st = particles.draw(dataclasses.replace(spec, x_margin=m), setup)
                xs = [torch.from_numpy(st[k]).to(device) for k in ("x", "y", "z")]
                g = [tmp.interp_lag3(c, *xs).cpu().numpy() for c in range(6)]
                st["u"], st["v"], st["w"] = g[0], g[1], g[2]
                particles.body_half_vorticity(st, g[3], g[4], g[5])
                jobs.append(serving.Job(state=st, steps=steps, arrival_s=t, field=fid))
    jobs.sort(key=lambda j: j.arrival_s)
    field_bytes = sum((n + 3) * (n + 4) ** 2 * 8 * 4 for n, _ in w.fields)
    budget = w.hbm_budget - field_bytes
    total = sum(j.n for j in jobs)
    cap = int(min(budget / serving.BYTES_PER_PARTICLE, 1.5 * total))   # pool sized for the stream
    ctx = api.Context(w.setup(w.fields[0][0]), "mixed", max_particles=cap)
    ctx.set_fields({k: fields[0][k].contiguous() for k in api.FIELD_KEYS})
    for fid in range(1, len(w.fields)):
        assert ctx.add_field(w.fields[fid][0]) == fid
        ctx.set_fields({k: fields[fid][k].contiguous() for k in api.FIELD_KEYS}, slot=fid)
    del fields
    tune = None
    if not args.no_autotune:
        # launch grids tuned on the largest job's particles, which then leave again
        big = max(jobs, key=lambda j: j.n)
        ig = ctx.add_class({k: np.array(v, copy=True) for k, v in big.state.items()}, big.field)
        tune = ctx.autotune()
        ctx.remove_class(ig)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        summary = serving.serve(ctx, jobs, budget)
    clocks = clk.summary()
    ctx.close()
    value = summary["particle_steps_per_s"]
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([value], dtype=torch.float64, device=device)
        dist.all_reduce(t)
        value = float(t.item())
    if rank == 0:
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
                "steps": None, "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
                "config": {"workload": w.name, "precision": "mixed", "arrival_rate_per_s": w.rate_per_s,
                           "window_s": args.serve_seconds, "jobs": len(jobs), "particles": total,
                           "hbm_budget_bytes": budget, "dtime": w.dtime, "launch_grids": tune},
                "latency_p50_s": summary["latency_p50_s"], "latency_p99_s": summary["latency_p99_s"],
                "serving": summary, "clocks": clocks,
                "e2e": {"value": value, "unit": "particle-steps/s",
                        "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                        "note": "every job enters from and returns to host arrays"}}
        if not emit:
            return {"workload": w.name, "particle_steps_per_s": value,
                    "latency_p50_s": summary["latency_p50_s"], "latency_p99_s": summary["latency_p99_s"],
                    "jobs": len(jobs), "particles": total, "window_s": args.serve_seconds,
                    "arrival_rate_per_s": w.rate_per_s, "hbm_budget_bytes": budget, "launch_grids": tune,
                    "max_resident_jobs": summary.get("max_resident"), "clocks": clocks}
        print(json.dumps(line), flush=True)
    return None


# ---------------------------------------------------------------------------
def main():
    args = parse()
    from gazpart_b200 import config
    if args.workload == config.C5.name:
        if args.impl == "reference":
            if int(os.environ.get("RANK", "0")) == 0:
                print(json.dumps({"impl": "reference", "unavailable": "serving is a form of the GPU path; the "
                                  "CPU port is timed on single-ensemble workloads"}), flush=True)
            return
        rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        dist = None
        if world > 1:
            import torch
            import torch.distributed as dist
            from datetime import timedelta
            dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                    device_id=torch.device(f"cuda:{local}"))
        run_serving(args, rank, world, local)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    w = config.WORKLOADS[args.workload]
    precision = args.precision or ("mixed" if w.field_dtype == "f32" else "fp64")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        if isinstance(w, config.BatchedWorkload):
            print(json.dumps({"impl": "reference", "unavailable": "the CPU port is timed on single-ensemble "
                              "workloads; a batched workload is many of them"}), flush=True)
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        threads = os.cpu_count() or 1
        scale = 16 if w.grid >= 256 else 1
        max_emaj = workload_max_emaj(w)
        k = max(1, min(args.steps, 4))
        if args.warmup:
            time_cpu(w, 1, threads, scale, max_emaj)
        r = time_cpu(w, k, threads, scale, max_emaj)
        sample = (f"{r['n']} particles at the workload's density in a (L/{scale})^3 periodic box, "
                  f"collision boxes sized from the full workload ({r['nbox']} boxes), "
                  f"{r['candidates_per_step']} candidate pairs/step each solved by Levenberg-Marquardt "
                  f"as the reference does; {k} steps timed")
        line = {"impl": "reference", "metric": "particle-steps/s", "value": r["value"], "unit": "particle-steps/s",
                "n_gpus": args.gpus, "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * (r["t_adv"] + r["t_col"]),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": {"workload": w.name, "precision": "fp64 (reference)"},
                "cpu_baseline": {"value": r["value"], "unit": "particle-steps/s", "cores": threads,
                                 "kind": "port", "sample": sample},
                "e2e": {"value": r["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    from gazpart_b200 import api
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device(device))

    # the autotuner's trials (4 launches x 5 grids x 3 one-step graphs, then up to 5 overlap
    # choices x 3 eight-step graphs) and the three one-step graphs also move the particles
    # before the state is restored, and the statistics timing adds 24 steps
    run_steps = args.warmup + args.steps + 2 * (args.e2e_steps + 1) + AUTOTUNE_STEPS + 6 + 28
    setup, f, st = build_inputs(w, device, precision, run_steps, rank, world)
    batched = isinstance(st, list)
    max_emaj = float(st["emaj"].max()) if not batched else None
    ctx = make_context(setup, f, st, precision, device)
    n = ctx.n
    if args.contact_tail is not None:
        ctx.set_contact_tail(args.contact_tail)
    if args.grids:
        g = [int(v) for v in args.grids.split(",")]
        tune = dict(zip(("gather", "integrate", "bin", "search"), g[:4]))
        tune["overlap_gather"] = bool(g[4]) if len(g) > 4 else False
        tune["speculative_integrate"] = len(g) > 4 and g[4] == 2
        if len(g) > 5:
            tune["contact_tail"] = g[5]
        ctx.set_launch(tune)
    else:
        tune = None if args.no_autotune else ctx.autotune()
    ctx.raise_status("autotune")
    ctx.step(args.warmup)
    ctx.sync()
    ctx.raise_status("warm-up")
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        total_ms, phases, kps = ctx.step_timed(args.steps)
        # In a multi-step graph the gather of step s+1 overlaps step s's contact solves,
        # so its phase time spans both.  The first step of a graph gathers alone: one-step
        # graphs give the kernel's own duration for the roofline.
        singles = [ctx.step_timed(1)[1] for _ in range(3)]
        alone = sorted(ph["gather"] for ph in singles)[1]
        phases_alone = {k: sorted(ph[k] for ph in singles)[1] for k in singles[0]}
    clocks = clk.summary()
    ctx.raise_status("timed steps")
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms = reduce_max_ms(total_ms, dist, device)
    ms_per_step = total_ms / args.steps
    # a batched workload is split over the ranks (strong scaling): its particles are the
    # sum of the shares; a single ensemble is replicated (weak scaling)
    n_job = n * world
    if batched and dist:
        tot = torch.tensor([n], dtype=torch.int64, device=device)
        dist.all_reduce(tot)
        n_job = int(tot.item())
    value = n_job * args.steps / (total_ms / 1e3)

    # roofline of the HBM-bound kernel of the step: the stencil gather (the phase
    # timestamps around it bracket that one kernel on the library's stream)
    fbytes = 4 if precision == "mixed" else 8
    bpp = gather_bytes_per_particle(6, fbytes)
    peak, peak_kind = hbm_peak()
    achieved = bpp * n / (alone / 1e3) / 1e9
    tr = GATHER_TRAFFIC.get((w.name, precision))
    roofline = {"bound": "hbm", "kernel": "k_gather", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "bytes_per_launch": bpp * n, "bytes_per_particle": bpp, "kernel_ms": alone,
                "kernel_ms_source": "median of three one-step graphs run right after the timed region",
                "traffic": None if tr is None else tr[0] * n, "traffic_source": None if tr is None else tr[1],
                "traffic_gbs": None if tr is None else tr[0] * n / (alone / 1e3) / 1e9}

    # end to end through the C ABI with host buffers: H2D of the state, one step,
    # D2H of the state, every step
    pinned = {k: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy() for k in api.STATE_KEYS}
    ctx.download_into(pinned)
    ctx.sync()
    ctx.step(1)            # capture the one-step graph outside the timed loop
    ctx.sync()
    parts = {"h2d": 0.0, "step": 0.0, "d2h": 0.0}
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        ta = time.perf_counter()
        ctx.put_state(pinned)
        tb = time.perf_counter()
        ctx.step(1)
        ctx.sync()
        tc = time.perf_counter()
        ctx.download_into(pinned)
        td = time.perf_counter()
        parts["h2d"] += tb - ta
        parts["step"] += tc - tb
        parts["d2h"] += td - tc
    e2e_s = (time.perf_counter() - t0) / args.e2e_steps
    ctx.raise_status("e2e steps")
    bytes_state = 13 * 8 * n
    serial = {"value": n / e2e_s, "unit": "particle-steps/s", "h2d_bytes_per_step": bytes_state,
              "d2h_bytes_per_step": bytes_state, "ms_per_step": 1e3 * e2e_s,
              "ms_parts": {k: 1e3 * v / args.e2e_steps for k, v in parts.items()},
              "api": "gp_put_state + gp_step(1) + gp_download_state"}
    # the same step as one call (gp_step_host): the copies overlap the step where the data
    # allow; same bytes each way, same results bit for bit
    ctx.step_host(pinned)
    ctx.sync()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        ctx.step_host(pinned)
    e2e_s = (time.perf_counter() - t0) / args.e2e_steps
    ctx.raise_status("e2e one-call steps")
    e2e = {"value": n / e2e_s, "unit": "particle-steps/s", "h2d_bytes_per_step": bytes_state,
           "d2h_bytes_per_step": bytes_state, "ms_per_step": 1e3 * e2e_s, "api": "gp_step_host"}

    restart_io = None
    if rank == 0 and not batched and not args.no_io:
        restart_io = time_restart_io(ctx, n, pinned)
    stats = None
    if not batched and not args.no_stats:
        stats = time_stats(ctx)
        ctx.raise_status("statistics")
    live_fluid = None
    if rank == 0 and not batched and not args.no_dns:
        live_fluid = time_live_fluid(ctx, setup, f)

    plain = None
    mixed_vs_fp64 = None
    if not args.no_plain and precision == "mixed":
        ctx.close()
        del ctx
        torch.cuda.empty_cache()
        if rank == 0 and world == 1 and not batched:
            mixed_vs_fp64 = compare_mixed_fp64(w, device, 10, {k: v for k, v in (tune or {}).items()
                                                               if k in ("gather", "integrate", "bin", "search")})
        st2 = build_inputs(w, device, "fp64", run_steps)[2]
        pctx = make_context(setup, {k: v for k, v in f.items()}, st2, "fp64", device)
        ptune = None if args.no_autotune else pctx.autotune()
        pctx.step(max(1, args.warmup))
        pctx.sync()
        # the same graph length as the mixed value, so that both include one unoverlapped
        # first step in the same proportion
        tms, pph, _ = pctx.step_timed(args.steps)
        pctx.raise_status("fp64 steps")
        plain = {"value": n * args.steps / (tms / 1e3), "steps": args.steps, "ms_per_step": tms / args.steps,
                 "phase_ms": pph, "launch_grids": ptune}
        pctx.close()
        del pctx
        torch.cuda.empty_cache()
    else:
        ctx.close()
        del ctx
        torch.cuda.empty_cache()

    batched_line = serving_line = None
    if rank == 0 and world == 1 and not batched and not args.no_forms:
        batched_line = time_batched(args, device)
        serving_line = run_serving(args, 0, 1, local, emit=False)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not batched:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        threads = os.cpu_count() or 1
        scale = 16 if w.grid >= 256 else 1
        r = time_cpu(w, 2, threads, scale, max_emaj)
        r1 = time_cpu_one_thread(w, scale, max_emaj)
        cpu = {"value": r["value"], "unit": "particle-steps/s", "cores": threads, "kind": "port",
               "cpu_model": cpu_model(),
               "sample": f"{r['n']} particles at the workload's density in a (L/{scale})^3 periodic box, "
                         f"{r['candidates_per_step']} LM contact solves/step as the reference does, 2 steps",
               "one_thread": {"value": r1["value"], "unit": "particle-steps/s", "cores": 1,
                              "sample": f"the same {r1['n']} particles: the advance timed whole, the collision "
                                        f"phase timed on {r1['pairs_timed']} random candidate pairs of "
                                        f"{r1['candidates_per_step']} (one LM solve each) and scaled",
                              "advance_s": r1["t_adv"], "collision_s": r1["t_col"]},
               "reference_fortran_toolchain": reference_compilers()}

    if rank == 0:
        line = {"metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "strong" if batched else "weak", "vs_baseline": None,
                "dtype": "f64" if precision == "fp64" else "f32/f64",
                "data": "synthetic",
                "config": {"workload": w.name, "precision": precision, "particles_per_gpu": n, "particles": n_job,
                           "field": f"{w.grid}^3 x 6 {'f32' if fbytes == 4 else 'f64'}",
                           "parallelism": (f"classes sharded over {world} GPUs" if batched and world > 1
                                           else f"replicas x{world}"),
                           "l2": "inputs larger than L2 (state+field > 5 GB)",
                           "x_margin": x_margin_for(w, run_steps), "launch_grids": tune,
                           "volume_fraction": None if (batched and world > 1) else volume_fraction(st, setup),
                           "classes": len(st) if batched else 1},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "e2e_put_step_download": serial,
                "gpu_launches": kps * args.steps,
                "kernels_per_step": kps, "phase_ms": phases,
                "phase_note": phase_note(tune),
                "phase_ms_one_step_graphs": phases_alone,
                "clocks": clocks, "fp64_plain": plain,
                "mixed_over_fp64": None if plain is None else value / plain["value"],
                "mixed_vs_fp64": mixed_vs_fp64, "batched": batched_line, "serving": serving_line,
                "restart_io": restart_io, "stats": stats, "live_fluid": live_fluid}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
