"""One state split into bands (evp1d.bands) on the GPU.

A single GPU holds every band's handle.  Between subcycles the library's
pack kernels gather each band's boundary velocities into device buffers.
The buffers move by device copies, standing in for NCCL send/recv, and the
unpack kernels scatter them into the receiving bands' state.  The phases are
separated by host synchronisation, so no kernel waits on another.  The owned
parts, put back together, equal the single-domain oracle run bit for bit.
BandSolver (the per-rank driver) runs at world size 1.
"""
import numpy as np
import pytest
import torch

import evp1d
from evp1d import bands as B
from evp1d import synth
from test_gpu_parity import oracle_run

pytestmark = pytest.mark.gpu


def _same(res, ref, pr):
    for k in ("stress", "strintx", "strinty", "Cb"):
        a, b = np.asarray(res[k]), np.asarray(getattr(ref, k))
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), k
    for k in ("uvel", "vvel"):
        a, b = np.asarray(res[k])[: pr.na], getattr(ref, k)[: pr.na]
        assert np.array_equal(a.view(np.int64), b.view(np.int64)), k


def _outs(fs):
    return dict(stress=fs.stress, uvel=fs.uvel, vvel=fs.vvel, strintx=fs.strintx,
                strinty=fs.strinty, Cb=fs.Cb)


def solve_bands_one_gpu(pr, nbands, ndte, own_buffers=False):
    """own_buffers: pack into and unpack from the handles' own exchange
    buffers (evp1d_exchange_buffers) instead of caller buffers."""
    bs = B.split(pr, nbands)
    dev = torch.device("cuda", 0)
    hs, fss, sbuf, rbuf = [], [], [], []
    try:
        for b in bs:
            s = evp1d.EVP1D.from_problem(b.local, ndte=ndte)
            s.exchange_setup(b.send_idx(), b.recv_idx())
            fs = evp1d.FieldSet.from_problem(b.local)
            s.upload(fs)
            hs.append(s)
            fss.append(fs)
            ns, nr = 2 * len(b.send_idx()), 2 * len(b.recv_idx())
            if own_buffers:
                ps, pr_ = s.exchange_buffers()
                assert (ps != 0) == (ns > 0) and (pr_ != 0) == (nr > 0)
                sbuf.append(B.device_view(ps, ns, dev))
                rbuf.append(B.device_view(pr_, nr, dev))
            else:
                sbuf.append(torch.zeros(ns, dtype=torch.float64, device=dev))
                rbuf.append(torch.zeros(nr, dtype=torch.float64, device=dev))
        for _ in range(ndte):
            for s in hs:
                s.subcycles(1)
            for s, buf in zip(hs, sbuf):
                s.exchange_pack(0 if own_buffers else buf.data_ptr())
            for s in hs:
                s.synchronize()
            torch.cuda.synchronize()
            for b, buf in zip(bs, rbuf):
                rs = b.slices("recv")
                for q, (o, n) in rs.items():
                    so, sn = bs[q].slices("send")[b.index]
                    assert sn == n
                    buf[2 * o: 2 * (o + n)].copy_(sbuf[q][2 * so: 2 * (so + n)])
            torch.cuda.synchronize()
            for s, buf in zip(hs, rbuf):
                s.exchange_unpack(0 if own_buffers else buf.data_ptr())
        for s, fs in zip(hs, fss):
            s.download(fs)
    finally:
        for s in hs:
            s.finalize()
    return B.assemble(pr, bs, [_outs(fs) for fs in fss])


@pytest.mark.parametrize("nbands,own", [(2, False), (3, False), (6, False), (3, True)])
def test_bands_on_one_gpu_bitwise(oracle_mod, nbands, own):
    pr = synth.to_1d(synth.make_grid(131, 77, seed=9, ndte=13, curvilinear=True))
    _same(solve_bands_one_gpu(pr, nbands, 13, own_buffers=own), oracle_run(oracle_mod, pr, 13), pr)


def test_band_solver_world_size_one(oracle_mod):
    """The per-rank driver with one band (no peers): the whole problem, one
    subcycle per launch through run_band, on the handle's stream."""
    pr = synth.make_problem("grid400x300", nx=120, ny=90, ndte=9)
    band = B.split(pr, 1)[0]
    fs = evp1d.FieldSet.from_problem(band.local)
    with B.BandSolver(band, ndte=9) as bsol:
        bsol.run(9, fs)
    _same(B.assemble(pr, [band], [_outs(fs)]), oracle_run(oracle_mod, pr, 9), pr)


@pytest.mark.parametrize("graph_steps", [0, 4])
def test_band_solver_graphs_bitwise(oracle_mod, monkeypatch, graph_steps):
    """The band step captured in CUDA graphs of 4 steps (and, for
    comparison, eagerly): 11 and then 11 more subcycles of one upload, so
    that graphs are captured for both ping-pong parities and replayed, with
    eager steps between them.  Bit for bit the oracle's 22 subcycles."""
    monkeypatch.setattr(B.BandSolver, "GRAPH_STEPS", graph_steps)
    pr = synth.make_problem("grid400x300", nx=100, ny=80, ndte=22)
    band = B.split(pr, 1)[0]
    fs = evp1d.FieldSet.from_problem(band.local)
    with B.BandSolver(band, ndte=22) as bsol:
        bsol.upload(fs)
        bsol.subcycles(11)
        bsol.subcycles(11)
        bsol.s.download(fs)
        if graph_steps:
            assert bsol.graph_launches > 0
            assert set(bsol._graphs) == {0, 1}
    _same(B.assemble(pr, [band], [_outs(fs)]), oracle_run(oracle_mod, pr, 22), pr)


def test_exchange_setup_validation():
    pr = synth.to_1d(synth.make_grid(40, 30, seed=2, ndte=4))
    with evp1d.EVP1D.from_problem(pr, ndte=4) as s:
        for send, recv in (([0], []), ([pr.na + 1], []), ([], [pr.navel + 1]), ([], [3, 3])):
            with pytest.raises(evp1d.EVP1DError) as e:
                s.exchange_setup(send, recv)
            assert e.value.code == -1
        s.exchange_setup([], [])  # empty lists are allowed
        with pytest.raises(evp1d.EVP1DError):  # nothing uploaded yet
            s.exchange_pack(0)
    members = [synth.make_problem("grid400x300", nx=20, ny=15, seed=80 + i, ndte=4) for i in range(2)]
    with evp1d.EVP1D.batched(synth.concat(members), ndte=4) as s:
        with pytest.raises(evp1d.EVP1DError):
            s.exchange_setup([1], [])
