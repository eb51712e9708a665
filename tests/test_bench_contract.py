"""The bench's reference arm on CPU (bench.py --impl reference): one JSON
line with the contract's keys, and under torchrun only rank 0 works and
prints (the other ranks exit 0 without output)."""
import json
import os
import subprocess
import sys

from conftest import ROOT

ARGS = ["--impl", "reference", "--config", "grid400x300", "--ndte", "4", "--steps", "2",
        "--warmup", "1"]


def _run(env_extra):
    env = dict(os.environ, OMP_NUM_THREADS="4", **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + ARGS, env=env,
                          capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_one_contract_line():
    r = _run({})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["config"]["workload"].startswith("evp1d grid400x300")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.strip().startswith("{")]


def test_short_stepu_condition(monkeypatch):
    """The roofline's byte count follows the kernel's choice of stepu part:
    377 B when every Tbu is +0, every uvel_init/vvel_init finite and
    revp == 0, else 401 B."""
    import numpy as np
    from evp1d import synth, roofline
    pr = synth.make_problem("grid400x300", nx=40, ny=30, ndte=3)
    assert roofline.short_stepu(pr, 0.0)
    assert roofline.per_point_subcycle("fused-tile-tma", True) == 377
    assert roofline.per_point_subcycle("fused-tile-tma", False) == 401
    assert roofline.per_point_subcycle("fused-tile", True) == 401
    assert not roofline.short_stepu(pr, 1.0)
    q = pr.copy()
    q.f["Tbu"] = q.f["Tbu"].copy()
    q.f["Tbu"][3] = -0.0
    assert not roofline.short_stepu(q, 0.0)
    q = pr.copy()
    q.f["uvel_init"] = q.f["uvel_init"].copy()
    q.f["uvel_init"][5] = np.inf
    assert roofline.short_stepu(q, 0.0)  # defaulted: the call-start velocities
    assert not roofline.short_stepu(q, 0.0, explicit_init=True)
    monkeypatch.setenv("EVP1D_COMPACT", "0")
    assert not roofline.short_stepu(pr, 0.0)
