"""One state split over two processes that share the one GPU.

Each process holds its band's handle.  Between subcycles the processes
exchange the ghost velocities over gloo, through host tensors copied from
and to the handles' own device buffers (evp1d_exchange_buffers), using the
same loop as the GPU driver (evp1d.bands.run_band).  The processes take
turns on the GPU: all GPU work of one process (handle set-up, a subcycle with
its pack, an unpack, the download) is followed by a synchronize and a gloo
barrier before the other process starts its own.  So their kernels never run
at the same time, and none waits on another.  The owned results, gathered
on rank 0, equal the single-domain oracle run bit for bit.  Only NCCL itself
(2+ GPUs) stays untested here.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ORACLE, PKG

pytestmark = pytest.mark.gpu

NDTE = 9


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    for p in (PKG, ORACLE):
        sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    import evp1d
    from evp1d import bands as B, synth
    dev = torch.device("cuda", 0)

    def in_turn(fn):
        """Run fn's GPU work while the other processes wait."""
        for r in range(world):
            if r == rank:
                fn()
                torch.cuda.synchronize()
            dist.barrier()

    pr = synth.to_1d(synth.make_grid(131, 77, seed=9, ndte=NDTE, curvilinear=True))
    band = B.split(pr, world)[rank]
    ns, nr = len(band.send_idx()), len(band.recv_idx())
    st = {}

    def setup():
        s = evp1d.EVP1D.from_problem(band.local, ndte=NDTE)
        s.exchange_setup(band.send_idx(), band.recv_idx())
        ps, pr_ = s.exchange_buffers()
        st.update(s=s, fs=evp1d.FieldSet.from_problem(band.local),
                  dsend=B.device_view(ps, 2 * ns, dev), drecv=B.device_view(pr_, 2 * nr, dev))
        s.upload(st["fs"])
        s.synchronize()

    in_turn(setup)
    s = st["s"]
    send = torch.zeros(2 * ns, dtype=torch.float64)
    recv = torch.zeros(2 * nr, dtype=torch.float64)

    def subcycle_and_pack():
        s.subcycles(1)
        s.exchange_pack()
        s.synchronize()
        send.copy_(st["dsend"].cpu())

    def unpack_from_host():
        st["drecv"].copy_(recv.to(dev))
        torch.cuda.synchronize()
        s.exchange_unpack()
        s.synchronize()

    B.run_band(band, NDTE, lambda: in_turn(subcycle_and_pack), lambda b: None,
               lambda b: in_turn(unpack_from_host), send, recv)
    in_turn(lambda: s.download(st["fs"]))
    fs = st["fs"]
    out = dict(stress=fs.stress, uvel=fs.uvel, vvel=fs.vvel, strintx=fs.strintx,
               strinty=fs.strinty, Cb=fs.Cb)
    in_turn(s.finalize)
    outs = [None] * world
    dist.all_gather_object(outs, out)
    if rank == 0:
        import oracle
        from test_bands import _same
        res = B.assemble(pr, B.split(pr, world), outs)
        try:
            _same(res, oracle.run_1d(pr, NDTE), pr)
            q.put("ok")
        except AssertionError as e:
            q.put(f"mismatch: {e}")
    dist.barrier()
    dist.destroy_process_group()


def test_two_processes_share_the_gpu_in_turns():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        assert q.get(timeout=300) == "ok"
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
