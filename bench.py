#!/usr/bin/env python
"""Benchmark of the EVP-1D subcycle loop (stress + stepu, ndte subcycles).

Metric: ice-point-subcycles/s (FP64) = active 1D points x subcycles / time,
over the whole job (all ranks).  One step = one dyn_evp1d_run-equivalent
call: ndte subcycles over one synthetic state of the operational-scale
configuration (1600 x 1200 grid, ~1.2M ice points, ndte = 1000).

  value   device-resident: state already in HBM, evp1d_subcycles(ndte) timed
          with CUDA events on the solver's stream.
  e2e     the same metric through evp1d_run with host buffers: upload,
          subcycles and download inside the timed region.
  roofline  algorithmic bytes of the fused subcycle / its measured duration,
          against the measured HBM copy bandwidth.
  cpu_baseline  the oracle's OpenMP SPMD port of the reference's v2b loop
          (f1 flags) on this host's cores, on a bounded sample.

--impl reference times that CPU path alone (rank 0) on the same workload.
Multi-GPU (torchrun): every rank solves its own independent state (an
ensemble member, seed + rank); no collective in the data path ("weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "cice-evp1d_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

# the CPU baseline's OpenMP threads stay on their cores (read by libgomp when
# the oracle library is first loaded)
os.environ.setdefault("OMP_PROC_BIND", "close")
os.environ.setdefault("OMP_PLACES", "cores")

METRIC = "EVP ice-point-subcycles/s (FP64)"
UNIT = "ice-point-subcycles/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", default="grid1600x1200")
    ap.add_argument("--ndte", type=int, default=None)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--split", action="store_true",
                    help="one state of --config split into one band per rank, with a "
                         "velocity exchange (NCCL) every subcycle: strong scaling")
    ap.add_argument("--band-timing", type=int, nargs="*", default=None,
                    help="time the bands of a split of --config into each given number "
                         "of bands on one GPU (the per-rank compute of such a split)")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave out the ensemble and adjoint keys of the default line")
    ap.add_argument("--extras-ndte", type=int, default=None,
                    help="subcycles of the ensemble and adjoint keys (default: the "
                         "configurations' own, 500)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_id}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# CPU: the oracle's OpenMP port of the reference loop
# --------------------------------------------------------------------------
def cpu_rate(pr, ndte_params: int, target_s: float, flavour: str = "f1"):
    """Time the oracle's SPMD OpenMP loop (src/evp_v2b.F90:91-110) on `pr`
    for a bounded number of subcycles.  Returns (rate, threads, n_sub, secs)."""
    import oracle
    p = oracle.params(ndte_params)
    st = oracle.State1D(pr)
    threads = os.cpu_count() or 1
    oracle.run_1d(pr, 1, p=p, mode="omp", flavour=flavour, nthreads=threads, state=st)
    t0 = time.perf_counter()
    oracle.run_1d(pr, 1, p=p, mode="omp", flavour=flavour, nthreads=threads, state=st)
    t1 = time.perf_counter() - t0
    n = max(1, min(ndte_params, int(target_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    oracle.run_1d(pr, n, p=p, mode="omp", flavour=flavour, nthreads=threads, state=st)
    dt = time.perf_counter() - t0
    return pr.n_active * n / dt, threads, n, dt


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def run_reference(args, rank, world):
    """--impl reference: the CPU port of the reference's loop, rank 0 only."""
    if rank != 0:
        return
    from evp1d import synth
    pr = synth.make_problem(args.config, **({"ndte": args.ndte} if args.ndte else {}))
    ndte = pr.ndte
    import oracle
    p = oracle.params(ndte)
    st = oracle.State1D(pr)
    threads = os.cpu_count() or 1
    # sample size per step: ~3 s of CPU work, at most ndte subcycles
    t0 = time.perf_counter()
    oracle.run_1d(pr, 1, p=p, mode="omp", nthreads=threads, state=st)
    t1 = time.perf_counter() - t0
    n_sub = max(1, min(ndte, int(3.0 / max(t1, 1e-6))))
    for _ in range(args.warmup):
        oracle.run_1d(pr, n_sub, p=p, mode="omp", nthreads=threads, state=st)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.run_1d(pr, n_sub, p=p, mode="omp", nthreads=threads, state=st)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = pr.n_active * n_sub * args.steps / tot
    sample = (f"{args.config}: {pr.n_active} points x {n_sub} subcycles per step "
              f"(of ndte={ndte}), OpenMP SPMD static split, f1 flags "
              f"(-O1 -fno-tree-vectorize -ffp-contract=off), {cpu_model()}")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, reference value ranges)",
        "config": workload_config(args.config, pr, ndte),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(name, pr, ndte):
    return {"workload": f"evp1d {name}: {pr.na} list points ({pr.n_active} active), "
                        f"navel={pr.navel}, ndte={ndte}, FP64",
            "na": pr.na, "navel": pr.navel, "active_points": pr.n_active,
            "ndte": ndte, "l2": "inputs larger than L2 (no flush needed)",
            "parallelism": "one independent state per GPU"}


# --------------------------------------------------------------------------
# GPU: ensemble (batched) configuration
# --------------------------------------------------------------------------
def run_ensemble(args, rank, world, local):
    """The 64-member ensemble: one batched handle (all members' tiles in one
    launch per subcycle) against looping one handle per member.  Under
    torchrun the members are split over the ranks (evp1d.ensemble.partition,
    balanced by point count; no data-path collective), each rank solving its
    share in one batched handle: strong scaling of the fixed ensemble, timed
    as the slowest rank."""
    import torch
    import evp1d
    from evp1d import synth, roofline as alg_bytes
    from evp1d.ensemble import partition

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    cfg = dict(synth.ENSEMBLES[args.config])
    if args.ndte:
        cfg["ndte"] = args.ndte
    everyone = synth.make_ensemble(**cfg)
    ndte = cfg["ndte"]
    mine = partition([m.n_active for m in everyone], world)[rank]
    members = [everyone[i] for i in mine]
    units_all = sum(m.n_active for m in everyone) * ndte
    ens = synth.concat(members)
    fs = evp1d.FieldSet.from_problem(ens.combined)
    s = evp1d.EVP1D.batched(ens, ndte=ndte, device=local)
    stream = torch.cuda.ExternalStream(s.stream, device=local)
    s.upload(fs)
    tuned = s.autotune(10)
    for _ in range(args.warmup):
        s.subcycles(ndte)
    s.synchronize()

    def slowest(t):
        if pg:
            x = torch.tensor([t], device="cuda", dtype=torch.float64)
            pg.all_reduce(x, op=pg.ReduceOp.MAX)
            t = float(x.item())
        return t

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    s.launch_count(reset=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.subcycles(ndte)
    e1.record(stream)
    e1.synchronize()
    s.synchronize()
    launches = s.launch_count()
    t_b = slowest(e0.elapsed_time(e1) / 1000.0)
    path = s.path
    s.finalize()
    # loop of single-member handles over this rank's members
    handles = []
    for m in members:
        h = evp1d.EVP1D.from_problem(m, ndte=ndte, device=local)
        h.upload(evp1d.FieldSet.from_problem(m))
        h.subcycles(ndte)
        h.synchronize()
        handles.append(h)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for h in handles:
            h.subcycles(ndte)
    for h in handles:
        h.synchronize()
    t_l = slowest(time.perf_counter() - t0)
    for h in handles:
        h.finalize()
    value = units_all * args.steps / t_b
    loop_value = units_all * args.steps / t_l
    short = all(alg_bytes.short_stepu(m, _params_revp(ndte)) for m in members)
    ab = alg_bytes.per_point_subcycle(path, short)
    units_rank = sum(m.n_active for m in members) * ndte
    achieved = ab * (units_rank / ndte) / (t_b / (args.steps * ndte)) / 1e9
    peak, peak_src = alg_bytes.hbm_peak(ROOT)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC + " (ensemble)", "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t_b / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, reference value ranges)",
            "config": {"workload": f"evp1d {args.config}: {len(everyone)} members, "
                                   f"{units_all // ndte} active points, ndte={ndte}, FP64",
                       "members": len(everyone), "active_points": units_all // ndte,
                       "member_points_min": int(min(m.n_active for m in everyone)),
                       "member_points_max": int(max(m.n_active for m in everyone)),
                       "members_on_rank0": len(members),
                       "ndte": ndte, "l2": "inputs larger than L2 (no flush needed)",
                       "parallelism": f"members split over {world} rank(s)"},
            "loop_value": loop_value, "batched_vs_loop": value / loop_value,
            "autotune": tuned,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                         "algorithmic_bytes_per_point_subcycle": ab, "kernel": path,
                         "note": "rank 0's share over the slowest rank's time"},
            "gpu_launches": launches,
        }), flush=True)
    if pg:
        pg.destroy_process_group()


# --------------------------------------------------------------------------
# GPU: adjoint configurations
# --------------------------------------------------------------------------
ADJ_METRIC = "EVP adjoint ice-point-subcycles/s (FP64)"


def _misfit_seed(u, v, uobs, vobs):
    return 2.0 * (u - uobs), 2.0 * (v - vobs)


def _timed(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1000.0


def _adjoint_once(s, stream, ndte, interval, lam, fields):
    """One gradient from the initial state: upload (untimed), the recording
    forward, then seed + reverse sweep, each timed with CUDA events on the
    solver's stream."""
    s.upload(fields())
    t_rec = _timed(stream, lambda: s.record_subcycles(ndte, interval))
    s.adjoint_seed(*lam)
    t_sw = _timed(stream, s.adjoint_sweep)
    s.synchronize()
    return t_rec, t_sw


def run_adjoint(args, rank, world, local):
    """Single-problem adjoint (800 x 600, ndte = 500, J = misfit of the final
    velocities, checkpoints every 50 subcycles): forward, recording forward and
    reverse sweep timed on the device; a finite-difference check along 32
    random directions (8 per gradient field)."""
    import numpy as np
    import torch
    import evp1d
    from evp1d import synth

    torch.cuda.set_device(local)
    over = {"ndte": args.ndte} if args.ndte else {}
    seed = synth.CONFIGS[args.config]["seed"] + 1000 * rank
    pr = synth.make_problem(args.config, seed=seed, **over)
    ndte = pr.ndte
    uobs, vobs = synth.observations(pr.na, seed=seed + 500)
    interval = synth.ADJOINT_INTERVAL
    fs = evp1d.FieldSet.from_problem(pr)
    s = evp1d.EVP1D.from_problem(pr, ndte=ndte, device=local)
    stream = torch.cuda.ExternalStream(s.stream, device=local)
    # final velocities for the seed of the misfit
    s.run_checkpointed(ndte, fs, interval)
    lam = _misfit_seed(fs.uvel[: pr.na], fs.vvel[: pr.na], uobs, vobs)
    fields = lambda: evp1d.FieldSet.from_problem(pr)
    s.upload(fields())
    for _ in range(args.warmup):
        s.subcycles(ndte)
        _adjoint_once(s, stream, ndte, interval, lam, fields)
        # the memory-sized recording too: its larger store is allocated here,
        # not in the timed steps
        _adjoint_once(s, stream, ndte, 0, lam, fields)
    s.upload(fields())
    props = torch.cuda.get_device_properties(local)
    gpu_id = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local)
    sampler = ClockSampler(gpu_id) if not args.no_clocks else None
    if sampler:
        sampler.__enter__()
    t_fwd, t_rec, t_sw, t_rec0, t_sw0 = [], [], [], [], []
    s.launch_count(reset=True)
    for _ in range(args.steps):
        t_fwd.append(_timed(stream, lambda: s.subcycles(ndte)))
        a, b = _adjoint_once(s, stream, ndte, interval, lam, fields)
        t_rec.append(a)
        t_sw.append(b)
        a, b = _adjoint_once(s, stream, ndte, 0, lam, fields)   # sized to memory
        t_rec0.append(a)
        t_sw0.append(b)
        s.upload(fields())
    launches = s.launch_count()
    if sampler:
        sampler.__exit__(None, None, None)
    s.upload(fields())
    s.record_subcycles(ndte, 0)
    info0 = s.adjoint_info()
    s.upload(fields())
    s.record_subcycles(ndte, interval)
    info = s.adjoint_info()
    s.adjoint_seed(*lam)
    s.adjoint_sweep()
    g = s.adjoint_gradients(("strength", "Cw", "forcex", "forcey"))

    # finite differences of the bit-exact forward, 32 directions
    rng = np.random.default_rng(seed + 7)
    h = 1e-6
    na = pr.na

    def run(prx):
        f = evp1d.FieldSet.from_problem(prx)
        s.run(ndte, f)
        return f.uvel[:na].copy(), f.vvel[:na].copy()

    def central(k, d, step):
        """Central difference of J along d, and the adjoint's derivative
        along the perturbation the two runs actually received (the rounded
        x +- step*d), both divided by 2 step."""
        prp, prm = pr.copy(), pr.copy()
        prp.f[k] = pr.f[k] + step * d
        prm.f[k] = pr.f[k] - step * d
        up, vp = run(prp)
        um, vm = run(prm)
        # summed point by point so that the difference does not cancel
        # against the size of J
        fd_ = float(np.sum((up - um) * (up + um - 2 * uobs) +
                           (vp - vm) * (vp + vm - 2 * vobs))) / (2 * step)
        ad_ = float(np.dot(g[k], prp.f[k] - prm.f[k])) / (2 * step)
        return fd_, ad_

    # central differences at relative steps 1e-4 .. 1e-7, 8 directions per
    # field: truncation error falls with the step, rounding error grows, and
    # the best step shows how close the adjoint is
    steps = (1e-4, 1e-5, 1e-6, 1e-7)
    fd = {k: {str(st_): 0.0 for st_ in steps} for k in ("strength", "Cw", "forcex", "forcey")}
    errs_h = {k: [] for k in fd}  # every direction's error at the step h
    for k in fd:
        for _ in range(8):
            d = pr.f[k] * rng.standard_normal(na)
            for st_ in steps:
                fd_, ad_ = central(k, d, st_)
                e = abs(fd_ - ad_) / abs(ad_)
                fd[k][str(st_)] = max(fd[k][str(st_)], e)
                if st_ == h:
                    errs_h[k].append(e)
    fd_err = {k: v[str(h)] for k, v in fd.items()}
    fd_best = {k: min(v.values()) for k, v in fd.items()}
    all_h = [e for v in errs_h.values() for e in v]
    fd_dirs = {"median_rel_err": float(np.median(all_h)),
               "within_1e-6": int(sum(e <= 1e-6 for e in all_h)), "of": len(all_h),
               "by_field": {k: sorted(v) for k, v in errs_h.items()}}
    s.finalize()

    med = statistics.median
    units = pr.n_active * ndte
    if rank == 0:
        print(json.dumps({
            "metric": ADJ_METRIC, "value": units / med(t_sw), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * med(t_sw), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, reference value ranges)",
            "config": dict(workload_config(args.config, pr, ndte),
                           loss="J = sum (u-u_obs)^2 + (v-v_obs)^2, u_obs, v_obs ~ N(0, 0.1)",
                           gradients="strength, Cw, forcex, forcey",
                           checkpoint_interval=interval),
            "forward_ms": 1000.0 * med(t_fwd),
            "record_ms": 1000.0 * med(t_rec),
            "sweep_ms": 1000.0 * med(t_sw),
            "adjoint_over_forward": med(t_sw) / med(t_fwd),
            "gradient_over_forward": (med(t_rec) + med(t_sw)) / med(t_fwd),
            "memory_sized": {"tape_subcycles": info0["tape_subcycles"],
                             "interval": info0["interval"],
                             "record_ms": 1000.0 * med(t_rec0),
                             "sweep_ms": 1000.0 * med(t_sw0),
                             "adjoint_over_forward": med(t_sw0) / med(t_fwd),
                             "store_bytes": info0["store_bytes"]},
            "memory_bytes": {"checkpoints_and_tape": info["store_bytes"],
                             "adjoint_work": info["work_bytes"],
                             "forward_solver": info["solver_bytes"]},
            "fd_check": {"directions": 32, "step": h, "max_rel_err": fd_err,
                         "directions_at_step": fd_dirs,
                         "max_rel_err_by_step": fd, "best_step_max_rel_err": fd_best},
            "gpu_launches": launches,
            "clocks": sampler.summary() if sampler else None,
        }), flush=True)


def run_adjoint_batched(args, rank, world, local):
    """The 32-member adjoint ensemble (ny = 600, nx ~ U(300, 1300), ndte =
    1000, gradients of the misfit with respect to forcex and forcey):
    one batched handle with memory-sized checkpoints against looping the
    single-member adjoint; gradients compared member by member."""
    import numpy as np
    import torch
    import evp1d
    from evp1d import synth

    torch.cuda.set_device(local)
    cfg = dict(synth.ENSEMBLES[args.config])
    if args.ndte:
        cfg["ndte"] = args.ndte
    cfg["seed"] += 1000 * rank
    members = synth.make_ensemble(**cfg)
    ndte = cfg["ndte"]
    ens = synth.concat(members)
    obs = [synth.observations(m.na, seed=cfg["seed"] + 500 + i) for i, m in enumerate(members)]
    want = ("forcex", "forcey")
    free0 = torch.cuda.mem_get_info(local)[0]
    fs = evp1d.FieldSet.from_problem(ens.combined)
    s = evp1d.EVP1D.batched(ens, ndte=ndte, device=local)
    stream = torch.cuda.ExternalStream(s.stream, device=local)
    s.run_checkpointed(ndte, fs, 0)
    u_list = np.concatenate([u[: m.na] for u, m in zip(ens.split_slots(fs.uvel), members)])
    v_list = np.concatenate([v[: m.na] for v, m in zip(ens.split_slots(fs.vvel), members)])
    uobs = np.concatenate([o[0] for o in obs])
    vobs = np.concatenate([o[1] for o in obs])
    lam = _misfit_seed(u_list, v_list, uobs, vobs)
    fields = lambda: evp1d.FieldSet.from_problem(ens.combined)
    for _ in range(args.warmup):
        _adjoint_once(s, stream, ndte, 0, lam, fields)
    t_rec, t_sw = [], []
    s.launch_count(reset=True)
    for _ in range(args.steps):
        a, b = _adjoint_once(s, stream, ndte, 0, lam, fields)
        t_rec.append(a)
        t_sw.append(b)
    launches = s.launch_count()
    peak_used = free0 - torch.cuda.mem_get_info(local)[0]
    info = s.adjoint_info()
    g = s.adjoint_gradients(want)
    s.finalize()
    # loop: one handle per member, the same work one member at a time
    loop_rec = loop_sw = 0.0
    worst = 0.0
    off = 0
    loop_peak = 0
    for i, m in enumerate(members):
        f1 = evp1d.FieldSet.from_problem(m)
        h = evp1d.EVP1D.from_problem(m, ndte=ndte, device=local)
        st = torch.cuda.ExternalStream(h.stream, device=local)
        h.run_checkpointed(ndte, f1, 0)
        lam_m = _misfit_seed(f1.uvel[: m.na], f1.vvel[: m.na], obs[i][0], obs[i][1])
        fm = lambda m=m: evp1d.FieldSet.from_problem(m)
        ts = [_adjoint_once(h, st, ndte, 0, lam_m, fm) for _ in range(args.steps)]
        loop_rec += statistics.median([t[0] for t in ts])
        loop_sw += statistics.median([t[1] for t in ts])
        gi = h.adjoint_gradients(want)
        inf = h.adjoint_info()
        loop_peak = max(loop_peak, inf["store_bytes"] + inf["work_bytes"] + inf["solver_bytes"])
        for k in want:
            ref = gi[k]
            worst = max(worst, float(np.abs(g[k][off: off + m.na] - ref).max()
                                     / max(np.abs(ref).max(), 1e-300)))
        h.finalize()
        off += m.na
    med = statistics.median
    units = sum(m.n_active for m in members) * ndte
    if rank == 0:
        print(json.dumps({
            "metric": ADJ_METRIC + " (ensemble)", "value": units / (med(t_rec) + med(t_sw)),
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * (med(t_rec) + med(t_sw)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, reference value ranges)",
            "config": {"workload": f"evp1d {args.config}: {len(members)} members, "
                                   f"{units // ndte} active points, ndte={ndte}, FP64 adjoint",
                       "members": len(members), "active_points": units // ndte,
                       "ndte": ndte, "gradients": "forcex, forcey",
                       "checkpoints": "sized to device memory"},
            "record_ms": 1000.0 * med(t_rec), "sweep_ms": 1000.0 * med(t_sw),
            "loop_record_ms": 1000.0 * loop_rec, "loop_sweep_ms": 1000.0 * loop_sw,
            "batched_vs_loop": (loop_rec + loop_sw) / (med(t_rec) + med(t_sw)),
            "max_rel_diff_vs_loop": worst,
            "checkpointing": {"tape_subcycles": info["tape_subcycles"],
                              "interval": info["interval"],
                              "checkpoints": info["checkpoints"]},
            "memory_bytes": {"checkpoints_and_tape": info["store_bytes"],
                             "adjoint_work": info["work_bytes"],
                             "forward_solver": info["solver_bytes"],
                             "device_used_peak": int(peak_used),
                             "loop_largest_member": loop_peak},
            "gpu_launches": launches,
        }), flush=True)


def run_split(args, rank, world, local):
    """--split: ONE state of the configuration split into `world` bands of
    the 1D list, one per rank (evp1d.bands).  Each rank solves its band and
    the band's forward ring; after every subcycle the ghost velocities move
    between the bands by NCCL send/recv (bands.run_band).  Strong scaling of
    the fixed state, timed on the device as the slowest rank.  The results
    are bit-identical to the single-domain run."""
    import torch
    import evp1d
    from evp1d import synth, bands, roofline as alg_bytes

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    over = {"ndte": args.ndte} if args.ndte else {}
    pr = synth.make_problem(args.config, **over)
    ndte = pr.ndte
    band = bands.split(pr, world)[rank]
    bsol = bands.BandSolver(band, ndte=ndte, device=local)
    s = bsol.s
    stream = torch.cuda.ExternalStream(s.stream, device=local)
    sweep = bsol.subcycles

    def reduce(x, op):
        if pg:
            t = torch.tensor([float(x)], device="cuda", dtype=torch.float64)
            pg.all_reduce(t, op=op)
            x = float(t.item())
        return x

    MAX = pg.ReduceOp.MAX if pg else None
    SUM = pg.ReduceOp.SUM if pg else None
    bsol.upload(evp1d.FieldSet.from_problem(band.local))
    for _ in range(args.warmup):
        sweep(ndte)
    s.synchronize()
    props = torch.cuda.get_device_properties(local)
    gpu_id = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local)
    sampler = ClockSampler(gpu_id) if not args.no_clocks else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.__enter__()
    s.launch_count(reset=True)
    bsol.graph_launches = 0
    e0.record(stream)
    for _ in range(args.steps):
        sweep(ndte)
    e1.record(stream)
    e1.synchronize()
    # kernels issued directly plus those the band's CUDA graphs replayed
    launches = s.launch_count() + bsol.graph_launches
    if sampler:
        sampler.__exit__(None, None, None)
    t_dev = e0.elapsed_time(e1) / 1000.0
    t_max = reduce(t_dev, MAX)
    value = pr.n_active * ndte * args.steps / t_max
    # end to end: BandSolver.run on page-locked host arrays of the band
    e2e = []
    for _ in range(args.e2e_steps):
        fs_e = evp1d.FieldSet.from_problem(band.local, pinned=True)
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        bsol.run(ndte, fs_e)
        a1.record(stream)
        a1.synchronize()
        e2e.append(a0.elapsed_time(a1) / 1000.0)
    e2e_value = pr.n_active * ndte / reduce(statistics.median(e2e), MAX) if e2e else None
    h2d, d2h = alg_bytes.host_bytes(band.local)
    h2d, d2h = reduce(h2d, SUM), reduce(d2h, SUM)
    sent = reduce(16 * len(band.send_idx()), SUM)
    ring = reduce(band.local.na - band.n_own, SUM)
    ab = alg_bytes.per_point_subcycle(s.path, alg_bytes.short_stepu(band.local, _params_revp(ndte)))
    sub_s = t_dev / (args.steps * ndte)
    achieved = ab * band.local.na / sub_s / 1e9
    peak, peak_src = alg_bytes.hbm_peak(ROOT)
    path = s.path
    bsol.finalize()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC + " (one state split over ranks)", "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, reference value ranges)",
            "config": dict(workload_config(args.config, pr, ndte),
                           parallelism=f"one state in {world} band(s) of the 1D list, "
                                       f"one per rank, velocity exchange every subcycle",
                           ring_points=int(ring), exchange_bytes_per_subcycle=int(sent)),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                         "algorithmic_bytes_per_point_subcycle": ab, "kernel": path,
                         "note": "rank 0's band (owned and ring points) over its own time"},
            "e2e": {"value": e2e_value, "unit": UNIT, "host_memory": "page-locked",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": launches,
            "clocks": sampler.summary() if sampler else None,
        }), flush=True)
    if pg:
        pg.destroy_process_group()


# --------------------------------------------------------------------------
# GPU: the ensemble and adjoint keys of the default line
# --------------------------------------------------------------------------
def _event_pair():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _params_revp(ndte: int) -> float:
    """revp of the parameters the bench's handles run with (the defaults of
    evp1d_set_evp_parameters)."""
    import evp1d
    return float(evp1d.set_evp_parameters(ndte).revp)


def ensemble_extras(local: int, steps: int, ndte: int = None) -> dict:
    """The 64-member ensemble (ens64): one batched handle against looping one
    handle per member, all CUDA-event timed on the device.

    - batched: evp1d_subcycles(ndte) of the batched handle.
    - serial loop: member after member, each evp1d_subcycles(ndte) followed by
      a synchronize before the next member starts (the loop a host code
      runs); the members' device times summed.
    - concurrent loop: every member issued at once, each on its own handle's
      stream; from an event all the streams wait on to an event that waits
      on all of them.
    - two-kernel loop: member after member, each subcycle as the reference's
      GPU code runs it, a stress launch then a stepu launch over the
      member's list (evp1d_stress_only / evp1d_stepu_only, in place),
      replayed from CUDA graphs of 50 subcycles so that no host launch
      overhead counts; the members' device times summed.
    - e2e: evp1d_run with page-locked host buffers (upload, subcycles,
      download), the batched handle's one call against the members' calls
      one after the other.
    - equal: one call of ndte from the same starting state, every output
      array of every member bit for bit between the batched handle and the
      serial loop."""
    import numpy as np
    import torch
    import evp1d
    from evp1d import synth

    cfg = dict(synth.ENSEMBLES["ens64"])
    if ndte:
        cfg["ndte"] = ndte
    ndte = cfg["ndte"]
    members = synth.make_ensemble(**cfg)
    ens = synth.concat(members)
    units = sum(m.n_active for m in members) * ndte
    dev = torch.device("cuda", local)

    # batched
    fb = evp1d.FieldSet.from_problem(ens.combined)
    s = evp1d.EVP1D.batched(ens, ndte=ndte, device=local)
    st_b = torch.cuda.ExternalStream(s.stream, device=dev)
    s.upload(fb)
    s.subcycles(ndte)
    s.synchronize()
    t_b = []
    for _ in range(steps):
        e0, e1 = _event_pair()
        e0.record(st_b)
        s.subcycles(ndte)
        e1.record(st_b)
        e1.synchronize()
        t_b.append(e0.elapsed_time(e1) / 1000.0)
    # end to end from page-locked host buffers
    fe = evp1d.FieldSet.from_problem(ens.combined, pinned=True)
    t_be = []
    for _ in range(steps):
        fe.refill(ens.combined)
        torch.cuda.synchronize()
        e0, e1 = _event_pair()
        e0.record(st_b)
        s.run(ndte, fe)
        e1.record(st_b)
        e1.synchronize()
        t_be.append(e0.elapsed_time(e1) / 1000.0)
    del fe
    # equality pass, from the starting state
    fb = evp1d.FieldSet.from_problem(ens.combined)
    s.run(ndte, fb)
    s.finalize()

    handles, streams = [], []
    for m in members:
        h = evp1d.EVP1D.from_problem(m, ndte=ndte, device=local)
        handles.append(h)
        streams.append(torch.cuda.ExternalStream(h.stream, device=dev))
    equal = True
    off = 0
    us, vs = ens.split_slots(fb.uvel), ens.split_slots(fb.vvel)
    for i, (m, h) in enumerate(zip(members, handles)):
        fm = evp1d.FieldSet.from_problem(m)
        h.run(ndte, fm)
        sl = slice(off, off + m.na)
        pairs = ((fb.stress[:, sl], fm.stress), (us[i][: m.na], fm.uvel[: m.na]),
                 (vs[i][: m.na], fm.vvel[: m.na]), (fb.strintx[sl], fm.strintx),
                 (fb.strinty[sl], fm.strinty), (fb.Cb[sl], fm.Cb))
        for a, b in pairs:
            equal &= bool(np.array_equal(np.ascontiguousarray(a).view(np.int64),
                                         np.ascontiguousarray(b).view(np.int64)))
        off += m.na
        h.upload(evp1d.FieldSet.from_problem(m))
        h.subcycles(ndte)
        h.synchronize()

    # serial loop
    t_s = []
    for _ in range(steps):
        tot = 0.0
        for h, st in zip(handles, streams):
            e0, e1 = _event_pair()
            e0.record(st)
            h.subcycles(ndte)
            e1.record(st)
            h.synchronize()
            tot += e0.elapsed_time(e1) / 1000.0
        t_s.append(tot)
    # the same serial loop end to end, from page-locked host buffers
    fms = [evp1d.FieldSet.from_problem(m, pinned=True) for m in members]
    t_se = []
    for _ in range(steps):
        tot = 0.0
        for m, h, st, fm in zip(members, handles, streams, fms):
            fm.refill(m)
            e0, e1 = _event_pair()
            e0.record(st)
            h.run(ndte, fm)
            e1.record(st)
            h.synchronize()
            tot += e0.elapsed_time(e1) / 1000.0
        t_se.append(tot)
    del fms
    # the two-kernel loop: stress launch, stepu launch per subcycle
    G = 50
    t_2k = []
    graphs = []
    for h, st in zip(handles, streams):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(st):
            with torch.cuda.graph(g, stream=st):
                for _ in range(G):
                    h.stress_only(1)
                    h.stepu_only(1)
        graphs.append(g)
    for _ in range(steps):
        tot = 0.0
        for h, st, g in zip(handles, streams, graphs):
            e0, e1 = _event_pair()
            e0.record(st)
            # a graph replays on torch's current stream: the member's
            with torch.cuda.stream(st):
                for _ in range(ndte // G):
                    g.replay()
                for _ in range(ndte % G):
                    h.stress_only(1)
                    h.stepu_only(1)
            e1.record(st)
            h.synchronize()
            tot += e0.elapsed_time(e1) / 1000.0
        t_2k.append(tot)
    del graphs
    # concurrent loop
    side = torch.cuda.Stream(device=dev)
    t_c = []
    for _ in range(steps):
        torch.cuda.synchronize()
        e0, e1 = _event_pair()
        e0.record(side)
        ends = []
        for h, st in zip(handles, streams):
            st.wait_event(e0)
            h.subcycles(ndte)
            e = torch.cuda.Event()
            e.record(st)
            ends.append(e)
        for e in ends:
            side.wait_event(e)
        e1.record(side)
        e1.synchronize()
        t_c.append(e0.elapsed_time(e1) / 1000.0)
    for h in handles:
        h.finalize()
    med = statistics.median
    b, sl_, co = units / med(t_b), units / med(t_s), units / med(t_c)
    tk, be, se = units / med(t_2k), units / med(t_be), units / med(t_se)
    return {"config": "ens64", "members": len(members), "active_points": units // ndte,
            "ndte": ndte, "steps": steps,
            "batched": b, "serial_loop": sl_, "concurrent_loop": co,
            "two_kernel_loop": tk, "unit": UNIT,
            "batched_over_serial_loop": b / sl_, "batched_over_concurrent_loop": b / co,
            "batched_over_two_kernel_loop": b / tk,
            "e2e": {"batched": be, "serial_loop": se, "batched_over_serial_loop": be / se,
                    "host_memory": "page-locked"},
            "ms": {"batched": 1000 * med(t_b), "serial_loop": 1000 * med(t_s),
                   "concurrent_loop": 1000 * med(t_c), "two_kernel_loop": 1000 * med(t_2k),
                   "e2e_batched": 1000 * med(t_be), "e2e_serial_loop": 1000 * med(t_se)},
            "equal_bitwise_per_member": equal,
            "timing": "CUDA events on the device; serial loop = sum of the members' "
                      "device times, one member at a time"}


def adjoint_extras(local: int, steps: int, ndte: int = None) -> dict:
    """The single-problem adjoint (adjoint800x600: J = misfit of the final
    velocities, gradients with respect to strength, Cw, forcex, forcey):
    forward, recording forward and reverse sweep, CUDA-event timed, with
    checkpoints every 50 subcycles and with the checkpointing sized to device
    memory.  The cost of a gradient is (record + sweep) / forward."""
    import torch
    import evp1d
    from evp1d import synth

    over = {"ndte": ndte} if ndte else {}
    pr = synth.make_problem("adjoint800x600", **over)
    ndte = pr.ndte
    uobs, vobs = synth.observations(pr.na, seed=synth.CONFIGS["adjoint800x600"]["seed"] + 500)
    interval = synth.ADJOINT_INTERVAL
    fs = evp1d.FieldSet.from_problem(pr)
    s = evp1d.EVP1D.from_problem(pr, ndte=ndte, device=local)
    stream = torch.cuda.ExternalStream(s.stream, device=torch.device("cuda", local))
    s.run(ndte, fs)
    lam = _misfit_seed(fs.uvel[: pr.na], fs.vvel[: pr.na], uobs, vobs)
    fields = lambda: evp1d.FieldSet.from_problem(pr)
    s.upload(fields())
    s.subcycles(ndte)
    _adjoint_once(s, stream, ndte, interval, lam, fields)
    _adjoint_once(s, stream, ndte, 0, lam, fields)
    t_f, t_r, t_w, t_r0, t_w0 = [], [], [], [], []
    for _ in range(steps):
        s.upload(fields())
        t_f.append(_timed(stream, lambda: s.subcycles(ndte)))
        a, b = _adjoint_once(s, stream, ndte, interval, lam, fields)
        t_r.append(a)
        t_w.append(b)
        a, b = _adjoint_once(s, stream, ndte, 0, lam, fields)
        t_r0.append(a)
        t_w0.append(b)
    info0 = s.adjoint_info()
    s.finalize()
    med = statistics.median
    f = med(t_f)
    return {"config": "adjoint800x600", "active_points": pr.n_active, "ndte": ndte,
            "steps": steps, "forward_ms": 1000 * f,
            "every_50": {"record_ms": 1000 * med(t_r), "sweep_ms": 1000 * med(t_w),
                         "gradient_over_forward": (med(t_r) + med(t_w)) / f,
                         "sweep_over_forward": med(t_w) / f},
            "memory_sized": {"record_ms": 1000 * med(t_r0), "sweep_ms": 1000 * med(t_w0),
                             "gradient_over_forward": (med(t_r0) + med(t_w0)) / f,
                             "tape_subcycles": info0["tape_subcycles"],
                             "interval": info0["interval"]},
            "timing": "CUDA events on the solver's stream"}


def run_band_timing(args, local):
    """--band-timing K...: the per-rank work of a split of --config into K
    bands, measured on one GPU.  Each band's handle runs 200 steps of (one
    subcycle, pack, unpack) on its own stream, timed with CUDA events on that
    stream; the exchange between GPUs (NCCL) is not part of it.  `us`: every
    step launched on its own and ending a call; `graphed_us`: the steps
    replayed from CUDA graphs of GRAPH_STEPS steps that do not end the call,
    as BandSolver runs them.  One JSON line per K: microseconds per step of
    every band and the bytes each band sends per subcycle."""
    import torch
    import evp1d
    from evp1d import synth, bands

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pr = synth.make_problem(args.config)
    nsub, warmup = 200, 5
    G = bands.BandSolver.GRAPH_STEPS
    for nb in (args.band_timing or [1, 2, 4, 8]):
        out = dict(problem=args.config, na=pr.na, nbands=nb, us=[], graphed_us=[], points=[],
                   ring=[], send_bytes=[])
        for b in bands.split(pr, nb):
            with evp1d.EVP1D.from_problem(b.local, device=local) as s:
                s.exchange_setup(b.send_idx(), b.recv_idx())
                s.upload(evp1d.FieldSet.from_problem(b.local))
                stream = torch.cuda.ExternalStream(s.stream, device=dev)

                def step(inner=False):
                    if inner:
                        s.subcycles_inner(1)
                    else:
                        s.subcycles(1)
                    s.exchange_pack()
                    s.exchange_unpack()

                for _ in range(warmup):
                    step()
                s.synchronize()
                e0, e1 = _event_pair()
                e0.record(stream)
                for _ in range(nsub):
                    step()
                e1.record(stream)
                e1.synchronize()
                out["us"].append(1000.0 * e0.elapsed_time(e1) / nsub)
                # the step BandSolver replays: graphs of G steps whose
                # subcycles do not end the call (no NCCL transfer here)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.stream(stream):
                    with torch.cuda.graph(g, stream=stream):
                        for _ in range(G):
                            step(inner=True)
                # a graph replays on torch's current stream: the handle's
                with torch.cuda.stream(stream):
                    g.replay()
                s.synchronize()
                e0, e1 = _event_pair()
                e0.record(stream)
                with torch.cuda.stream(stream):
                    for _ in range(nsub // G):
                        g.replay()
                e1.record(stream)
                e1.synchronize()
                out["graphed_us"].append(1000.0 * e0.elapsed_time(e1) / (G * (nsub // G)))
                del g
                out["points"].append(b.n_own)
                out["ring"].append(b.local.na - b.n_own)
                out["send_bytes"].append(16 * len(b.send_idx()))
        out["max_us"] = max(out["us"])
        out["max_graphed_us"] = max(out["graphed_us"])
        if nb == 1:
            # the same one-band step through BandSolver (graphs of 50 steps)
            # against evp1d_subcycles of the band's problem
            b = bands.split(pr, 1)[0]
            with bands.BandSolver(b, device=local) as bsol:
                bsol.upload(evp1d.FieldSet.from_problem(b.local))
                stream = torch.cuda.ExternalStream(bsol.s.stream, device=dev)
                bsol.subcycles(100)
                bsol.s.synchronize()
                e0, e1 = _event_pair()
                e0.record(stream)
                bsol.subcycles(nsub)
                e1.record(stream)
                e1.synchronize()
                out["band_solver_graphed_us"] = 1000.0 * e0.elapsed_time(e1) / nsub
                e0, e1 = _event_pair()
                e0.record(stream)
                bsol.s.subcycles(nsub)
                e1.record(stream)
                e1.synchronize()
                out["evp1d_subcycles_us"] = 1000.0 * e0.elapsed_time(e1) / nsub
        print(json.dumps(out), flush=True)


# --------------------------------------------------------------------------
# GPU
# --------------------------------------------------------------------------
def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    from evp1d import synth as _synth
    if args.config == "adjoint800x600":
        run_adjoint(args, rank, world, local)
        return
    if args.config == "adjoint_ens32":
        run_adjoint_batched(args, rank, world, local)
        return
    if args.config in _synth.ENSEMBLES:
        run_ensemble(args, rank, world, local)
        return
    if args.split:
        run_split(args, rank, world, local)
        return
    if args.band_timing is not None:
        if rank == 0:
            run_band_timing(args, local)
        return

    import numpy as np
    import torch
    import evp1d
    from evp1d import synth
    from evp1d import roofline as alg_bytes

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist

    over = {"ndte": args.ndte} if args.ndte else {}
    seed = synth.CONFIGS[args.config]["seed"] + 1000 * rank
    pr = synth.make_problem(args.config, seed=seed, **over)
    ndte = pr.ndte
    fs = evp1d.FieldSet.from_problem(pr)
    solver = evp1d.EVP1D.from_problem(pr, ndte=ndte, device=local)
    stream = torch.cuda.ExternalStream(solver.stream, device=local)

    def barrier():
        if pg:
            pg.barrier()

    # ---------------- device-resident timing ----------------
    solver.upload(fs)
    for _ in range(args.warmup):
        solver.subcycles(ndte)
    solver.synchronize()
    props = torch.cuda.get_device_properties(local)
    gpu_id = f"GPU-{props.uuid}" if getattr(props, "uuid", None) else str(local)
    sampler = ClockSampler(gpu_id) if not args.no_clocks else None
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    if sampler:
        sampler.__enter__()
    solver.launch_count(reset=True)
    ev0.record(stream)
    for _ in range(args.steps):
        solver.subcycles(ndte)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    launches = solver.launch_count()
    if sampler:
        sampler.__exit__(None, None, None)
    barrier()
    t_dev = ev0.elapsed_time(ev1) / 1000.0
    t_max = t_dev
    if pg:
        t = torch.tensor([t_dev], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        t_max = float(t.item())
    # the ranks solve different seeded states: sum the points they processed
    n_active_all = pr.n_active
    if pg:
        t = torch.tensor([float(pr.n_active)], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.SUM)
        n_active_all = int(t.item())
    value = n_active_all * ndte * args.steps / t_max

    # ---------------- roofline of the subcycle ----------------
    short = alg_bytes.short_stepu(pr, _params_revp(ndte))
    ab = alg_bytes.per_point_subcycle(solver.path, short)
    sub_s = t_dev / (args.steps * ndte)
    achieved = ab * pr.n_active / sub_s / 1e9
    peak, peak_src = alg_bytes.hbm_peak(ROOT)

    # ---------------- lindividual: stress alone, stepu alone ----------------
    # the reference-order kernels of the lindividual loops (src/evp_v2b.F90:
    # 127-155), timed on the device-resident state
    n_ind = min(ndte, 200)

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1000.0

    solver.stress_only(2)
    solver.stepu_only(2)
    t_so = timed(lambda: solver.stress_only(n_ind))
    t_uo = timed(lambda: solver.stepu_only(n_ind))
    # algorithmic bytes per point: stress reads 7 inputs, 12 stresses and the
    # point's u, v, writes 12 stresses and 8 str, plus 3 indices and a flag;
    # stepu reads 14 inputs, u, v and 8 str, writes u, v, strintx, strinty,
    # Cb, plus 3 indices and a flag
    b_so, b_uo = 41 * 8 + 13, 29 * 8 + 13
    lind = {"subcycles": n_ind,
            "stress_only": pr.n_active * n_ind / t_so,
            "stepu_only": pr.n_active * n_ind / t_uo,
            "stress_bytes_per_point": b_so, "stepu_bytes_per_point": b_uo,
            "stress_frac": b_so * pr.n_active * n_ind / t_so / 1e9 / alg_bytes.hbm_peak(ROOT)[0],
            "stepu_frac": b_uo * pr.n_active * n_ind / t_uo / 1e9 / alg_bytes.hbm_peak(ROOT)[0]}

    # ---------------- end to end (host buffers) ----------------
    # inputs in page-locked host memory (evp1d_host_alloc), refilled with the
    # step's starting state before each timed call
    h2d, d2h = alg_bytes.host_bytes(pr)
    e2e_times = []
    fs_e = evp1d.FieldSet.from_problem(pr, pinned=True) if args.e2e_steps > 0 else None
    barrier()
    for _ in range(args.e2e_steps):
        fs_e.refill(pr)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.run(ndte, fs_e)
        e1.record(stream)
        e1.synchronize()
        e2e_times.append(e0.elapsed_time(e1) / 1000.0)
    e2e_value = None
    if e2e_times:
        t_e2e = statistics.median(e2e_times)
        if pg:
            t = torch.tensor([t_e2e], device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e_value = n_active_all * ndte / t_e2e

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, threads, n_sub, secs = cpu_rate(pr, ndte, args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{pr.n_active} points x {n_sub} subcycles ({secs:.1f} s), "
                         f"oracle OpenMP SPMD port of src/evp_v2b.F90:91-110, f1 flags, "
                         f"{threads} threads, OMP_PROC_BIND={os.environ.get('OMP_PROC_BIND')}, "
                         f"{cpu_model()}"}
        # the same loop built for speed (the reference's f2-like flags:
        # -O3 -march=x86-64-v3, FMA contraction allowed), for context
        rate2, _, n2, secs2 = cpu_rate(pr, ndte, args.cpu_seconds / 2, flavour="f2")
        cpu["f2"] = {"value": rate2, "flags": "-O3 -march=x86-64-v3 -fopenmp",
                     "sample": f"{pr.n_active} points x {n2} subcycles ({secs2:.1f} s)"}

    path = solver.path
    solver.finalize()
    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        extras["ensemble"] = ensemble_extras(local, 3, args.extras_ndte)
        extras["adjoint"] = adjoint_extras(local, 3, args.extras_ndte)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, reference value ranges)",
            "config": workload_config(args.config, pr, ndte),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": alg_bytes.measured_traffic(ROOT, path, args.config),
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_point_subcycle": ab,
                         "kernel": path,
                         "stepu_part": ("short: Tbu +0, uvel_init/vvel_init finite, revp 0"
                                        if short else "full"),
                         # the same rate over the full stepu part's 401 B, for
                         # comparison with calls that need it
                         "full_part_equivalent": {
                             "bytes_per_point_subcycle": alg_bytes.per_point_subcycle(path),
                             "equivalent_gbs": alg_bytes.per_point_subcycle(path) * pr.n_active / sub_s / 1e9,
                             "equivalent_frac": alg_bytes.per_point_subcycle(path) * pr.n_active / sub_s / 1e9 / peak},
                         # the same rate over the reference's unfused data
                         # contract (str1..8 through HBM, 576 B): what the
                         # reference's two kernels would have to move
                         "reference_contract": {
                             "bytes_per_point_subcycle": alg_bytes.per_point_subcycle("two-kernel"),
                             "equivalent_gbs": alg_bytes.per_point_subcycle("two-kernel") * pr.n_active / sub_s / 1e9,
                             "equivalent_frac": alg_bytes.per_point_subcycle("two-kernel") * pr.n_active / sub_s / 1e9 / peak}},
            "e2e": {"value": e2e_value, "unit": UNIT, "host_memory": "page-locked",
                    "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": sampler.summary() if sampler else None,
            "lindividual": lind,
            "cpu_baseline": cpu,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
