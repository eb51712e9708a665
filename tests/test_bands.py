"""One state split into bands of the 1D list (evp1d.bands), on CPU.

The bands' local problems are solved by the oracle one subcycle at a time,
with the velocity exchange between subcycles.  The owned parts, put back
together, must equal the single-domain oracle run bit for bit.  Also covered:
the consistency of the exchange lists, bands thinner than a grid row, empty
bands, and world-size-2 and world-size-3 gloo ranks that run
evp1d.bands.run_band (the loop the GPU solver uses) over the oracle.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ORACLE, PKG


def _oracle():
    import oracle
    return oracle


def _same(res, ref, pr):
    for k in ("stress", "strintx", "strinty", "Cb"):
        a, b = np.asarray(res[k]), np.asarray(getattr(ref, k))
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), k
    for k in ("uvel", "vvel"):
        a, b = res[k][: pr.na], getattr(ref, k)[: pr.na]
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), k


def _outs(st):
    return dict(stress=st.stress, uvel=st.uvel, vvel=st.vvel, strintx=st.strintx,
                strinty=st.strinty, Cb=st.Cb)


def solve_in_process(pr, nbands, ndte):
    """Every band by the oracle, the exchange as direct copies."""
    oracle = _oracle()
    from evp1d import bands as B
    p = oracle.params(ndte)
    bs = B.split(pr, nbands)
    sts = [oracle.State1D(b.local) for b in bs]
    for _ in range(ndte):
        for b, st in zip(bs, sts):
            if b.local.na:
                oracle.run_1d(b.local, 1, p=p, state=st)
        for b, st in zip(bs, sts):
            for q, pos in b.recvs.items():
                src = bs[q].sends[b.index] - 1
                st.uvel[pos - 1] = sts[q].uvel[src]
                st.vvel[pos - 1] = sts[q].vvel[src]
    return bs, B.assemble(pr, bs, [_outs(st) for st in sts])


def _grid(nx, ny, seed, ndte, curvilinear=False):
    from evp1d import synth
    return synth.to_1d(synth.make_grid(nx, ny, seed=seed, ndte=ndte, curvilinear=curvilinear))


@pytest.mark.parametrize("nbands", [1, 2, 3, 8])
def test_bands_bitwise_with_the_single_domain_run(nbands):
    pr = _grid(60, 40, 3, 12)
    _, res = solve_in_process(pr, nbands, 12)
    _same(res, _oracle().run_1d(pr, 12), pr)


def test_thin_bands_on_a_curvilinear_grid():
    """Bands of about 40 points, shorter than a grid row: a band's ring and
    ghosts reach two and more bands ahead and behind."""
    pr = _grid(131, 77, 9, 6, curvilinear=True)
    nb = pr.na // 40
    bs, res = solve_in_process(pr, nb, 6)
    assert max(len(b.recvs) for b in bs) >= 3
    _same(res, _oracle().run_1d(pr, 6), pr)


def test_more_bands_than_points():
    from evp1d import bands as B
    pr = _grid(6, 5, 11, 5)
    nb = pr.na + 3
    bs, res = solve_in_process(pr, nb, 5)
    assert sum(b.n_own == 0 for b in bs) == 3
    assert all(not b.sends and not b.recvs for b in bs if b.n_own == 0)
    _same(res, _oracle().run_1d(pr, 5), pr)
    with pytest.raises(ValueError):
        B.split(pr, 0)


def test_exchange_lists_are_consistent():
    """What band b receives from q is what q sends to b, point for point;
    senders send owned list points only; receivers receive into their ring
    and halo slots only, never into owned points."""
    from evp1d import bands as B
    pr = _grid(90, 50, 5, 4, curvilinear=True)
    bs = B.split(pr, 5)
    for b in bs:
        assert np.all(b.local.skipU[b.n_own:] == 1)
        assert np.array_equal(b.local.skipU[: b.n_own], pr.skipU[b.lo: b.hi])
        for q, pos in b.recvs.items():
            src = bs[q].sends[b.index]
            assert len(src) == len(pos) > 0
            assert np.array_equal(bs[q].gid[src - 1], b.gid[pos - 1])
            assert np.all(src <= bs[q].n_own)
            assert np.all(pos > b.n_own)
        assert set(b.sends) == {q for q in range(len(bs)) if b.index in bs[q].recvs}
        # buffer layout: peers in order, contiguous
        sl = b.slices("recv")
        assert sum(n for _, n in sl.values()) == len(b.recv_idx())


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, ndte, q):
    import sys
    for p in (PKG, ORACLE):
        sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import oracle
    from evp1d import bands as B
    pr = _grid(70, 45, 13, ndte)
    band = B.split(pr, world)[rank]
    p = oracle.params(ndte)
    st = oracle.State1D(band.local)
    si, ri = band.send_idx() - 1, band.recv_idx() - 1

    def pack(buf):
        buf[0::2] = torch.from_numpy(st.uvel[si])
        buf[1::2] = torch.from_numpy(st.vvel[si])

    def unpack(buf):
        st.uvel[ri] = buf[0::2].numpy()
        st.vvel[ri] = buf[1::2].numpy()

    send = torch.empty(2 * len(si), dtype=torch.float64)
    recv = torch.empty(2 * len(ri), dtype=torch.float64)
    dist.barrier()
    B.run_band(band, ndte, lambda: oracle.run_1d(band.local, 1, p=p, state=st), pack, unpack,
               send, recv)
    outs = [None] * world
    dist.all_gather_object(outs, _outs(st))
    if rank == 0:
        res = B.assemble(pr, B.split(pr, world), outs)
        ref = oracle.run_1d(pr, ndte)
        try:
            _same(res, ref, pr)
            q.put("ok")
        except AssertionError as e:
            q.put(f"mismatch: {e}")
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchange_through_run_band(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, 8, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        assert q.get(timeout=240) == "ok"
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
