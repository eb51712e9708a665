"""Ensemble members sharded over ranks: one process per GPU, each solving its
own members in one batched handle.  Members are independent, so the data path
has no collective; ranks only exchange small per-member summaries on the host
at the end (``all_gather_object``)."""
from __future__ import annotations

import heapq

import numpy as np


def partition(sizes, world: int) -> list:
    """Largest-first greedy split of members over ``world`` ranks balancing the
    summed point counts.  Returns per-rank sorted member index lists."""
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for m in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        load, r = heapq.heappop(heap)
        out[r].append(m)
        heapq.heappush(heap, (load + int(sizes[m]), r))
    return [sorted(x) for x in out]


def solve_on_gpu(members: list, ndte: int, device: int = 0) -> list:
    """Solve `members` in one batched handle on `device`; returns per member a
    dict of result arrays (stress, uvel, vvel, strintx, strinty, Cb)."""
    import evp1d
    from evp1d import synth
    ens = synth.concat(members)
    fs = evp1d.FieldSet.from_problem(ens.combined)
    with evp1d.EVP1D.batched(ens, ndte=ndte, device=device) as s:
        s.run(ndte, fs)
    out = []
    for m in range(len(members)):
        out.append(dict(stress=ens.split_points(fs.stress)[m].copy(),
                        uvel=ens.split_slots(fs.uvel)[m].copy(),
                        vvel=ens.split_slots(fs.vvel)[m].copy(),
                        strintx=ens.split_points(fs.strintx)[m].copy(),
                        strinty=ens.split_points(fs.strinty)[m].copy(),
                        Cb=ens.split_points(fs.Cb)[m].copy()))
    return out


def summarize(res: dict, na: int) -> dict:
    """Small host-side summary of one member's results: bitwise hashes of
    the two reference output files' worth of data."""
    import hashlib
    h1 = hashlib.md5(np.ascontiguousarray(res["stress"], dtype="<f8").tobytes()).hexdigest()
    h2 = hashlib.md5(b"".join(np.ascontiguousarray(np.asarray(res[k])[:na], dtype="<f8").tobytes()
                              for k in ("strintx", "strinty", "uvel", "vvel"))).hexdigest()
    return {"stress_md5": h1, "stepu_md5": h2}


def sharded_run(members: list, ndte: int, solve=None, group=None) -> dict:
    """Every rank solves its share of `members` (``solve(list, ndte) -> list of
    result dicts``, default: the GPU batched solver on this rank's device) and
    all ranks receive {member index: summary} for every member."""
    import torch.distributed as dist
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    mine = partition([m.na for m in members], world)[rank]
    if solve is None:
        import torch
        dev = torch.cuda.current_device() if torch.cuda.is_available() else 0
        solve = lambda ms, n: solve_on_gpu(ms, n, dev)  # noqa: E731
    results = solve([members[i] for i in mine], ndte) if mine else []
    local = {i: summarize(r, members[i].na) for i, r in zip(mine, results)}
    if world == 1:
        return local
    gathered = [None] * world
    dist.all_gather_object(gathered, local, group=group)
    merged = {}
    for g in gathered:
        merged.update(g)
    return merged
