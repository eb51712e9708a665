"""Ensemble sharding over ranks on CPU: world-size-2 gloo processes split the
members (no collective in the data path), each solves its share, and every
rank ends with the same summaries a single process computes."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ORACLE, PKG


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_solve(members, ndte):
    import oracle
    out = []
    for pr in members:
        st = oracle.run_1d(pr, ndte)
        out.append(dict(stress=st.stress, uvel=st.uvel[: pr.navel], vvel=st.vvel[: pr.navel],
                        strintx=st.strintx, strinty=st.strinty, Cb=st.Cb))
    return out


def _members():
    from evp1d import synth
    return [synth.make_problem("grid400x300", nx=nx, ny=30, seed=70 + i, ndte=4)
            for i, nx in enumerate([25, 60, 12, 44, 33])]


def _worker(rank, world, port, q):
    import sys
    for p in (PKG, ORACLE):
        sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from evp1d import ensemble
    res = ensemble.sharded_run(_members(), 4, solve=_oracle_solve)
    q.put((rank, res))
    dist.barrier()
    dist.destroy_process_group()


def test_partition_balances_and_covers():
    from evp1d import ensemble
    sizes = [100, 90, 80, 10, 10, 5, 1]
    parts = ensemble.partition(sizes, 3)
    assert sorted(sum(parts, [])) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    assert ensemble.partition([3], 4)[1:] == [[], [], []]


def test_two_ranks_match_single_process():
    from evp1d import ensemble
    want = ensemble.sharded_run(_members(), 4, solve=_oracle_solve)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, res in got:
        assert res == want, f"rank {rank} differs"
    assert len(want) == 5
