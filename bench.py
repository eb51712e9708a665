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

METRIC = "EVP ice-point-subcycles/s (FP64)"
UNIT = "ice-point-subcycles/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--config", default="cfg2")
    ap.add_argument("--ndte", type=int, default=None)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
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
    launch per subcycle) against looping one handle per member."""
    import torch
    import evp1d
    from evp1d import synth, roofline as alg_bytes

    torch.cuda.set_device(local)
    cfg = dict(synth.ENSEMBLES[args.config])
    if args.ndte:
        cfg["ndte"] = args.ndte
    cfg["seed"] += 1000 * rank
    members = synth.make_ensemble(**cfg)
    ndte = cfg["ndte"]
    ens = synth.concat(members)
    units = sum(m.n_active for m in members) * ndte
    fs = evp1d.FieldSet.from_problem(ens.combined)
    s = evp1d.EVP1D.batched(ens, ndte=ndte, device=local)
    stream = torch.cuda.ExternalStream(s.stream, device=local)
    s.upload(fs)
    tuned = s.autotune(10)
    for _ in range(args.warmup):
        s.subcycles(ndte)
    s.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.launch_count(reset=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.subcycles(ndte)
    e1.record(stream)
    e1.synchronize()
    s.synchronize()
    launches = s.launch_count()
    t_b = e0.elapsed_time(e1) / 1000.0
    path = s.path
    s.finalize()
    # loop of single-member handles on the same stream order
    handles = []
    for m in members:
        h = evp1d.EVP1D.from_problem(m, ndte=ndte, device=local)
        h.upload(evp1d.FieldSet.from_problem(m))
        h.subcycles(ndte)
        h.synchronize()
        handles.append(h)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for h in handles:
            h.subcycles(ndte)
    for h in handles:
        h.synchronize()
    t_l = time.perf_counter() - t0
    for h in handles:
        h.finalize()
    value = units * args.steps / t_b
    loop_value = units * args.steps / t_l
    ab = alg_bytes.per_point_subcycle(path)
    achieved = ab * (units / ndte) / (t_b / (args.steps * ndte)) / 1e9
    peak, peak_src = alg_bytes.hbm_peak(ROOT)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC + " (ensemble)", "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t_b / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, reference value ranges)",
            "config": {"workload": f"evp1d {args.config}: {len(members)} members, "
                                   f"{units // ndte} active points, ndte={ndte}, FP64",
                       "members": len(members), "active_points": units // ndte,
                       "member_points_min": int(min(m.n_active for m in members)),
                       "member_points_max": int(max(m.n_active for m in members)),
                       "ndte": ndte, "l2": "inputs larger than L2 (no flush needed)"},
            "loop_value": loop_value, "batched_vs_loop": value / loop_value,
            "autotune": tuned,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                         "algorithmic_bytes_per_point_subcycle": ab, "kernel": path},
            "gpu_launches": launches,
        }), flush=True)


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
    if args.config in _synth.ENSEMBLES:
        run_ensemble(args, rank, world, local)
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
    units_rank = pr.n_active * ndte * args.steps
    value = units_rank * world / t_max

    # ---------------- roofline of the subcycle ----------------
    ab = alg_bytes.per_point_subcycle(solver.path)
    sub_s = t_dev / (args.steps * ndte)
    achieved = ab * pr.n_active / sub_s / 1e9
    peak, peak_src = alg_bytes.hbm_peak(ROOT)

    # ---------------- end to end (host buffers) ----------------
    h2d, d2h = alg_bytes.host_bytes(pr)
    e2e_times = []
    barrier()
    for _ in range(args.e2e_steps):
        fs_e = evp1d.FieldSet.from_problem(pr)
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
        e2e_value = pr.n_active * ndte * world / t_e2e

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, threads, n_sub, secs = cpu_rate(pr, ndte, args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{pr.n_active} points x {n_sub} subcycles ({secs:.1f} s), "
                         f"oracle OpenMP SPMD port of src/evp_v2b.F90:91-110, f1 flags, "
                         f"{threads} threads, {cpu_model()}"}

    path = solver.path
    solver.finalize()
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
                         "kernel": path},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "clocks": sampler.summary() if sampler else None,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
