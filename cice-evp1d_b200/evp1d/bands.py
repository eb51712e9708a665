"""One state split over ranks in bands of the 1D list, with one velocity
exchange per subcycle.

The reference solves the whole domain in one process: CICE gathers the
global arrays onto the master task before the 1D solver runs
(gather_global_ext, integration/ice_dyn_evp1d.F90:637-716).  Here each rank
holds a band of the global list and solves it on its own GPU.

Band b owns the global list points [lo, hi) (j-outer, i-inner order, so a
band is a run of grid rows).  Its local 1D problem holds:
  - the owned points, first and in global order;
  - the forward ring G: list points outside the band that are stepu
    neighbours (nw, sw, sse) of owned points.  stepu of an owned point needs
    their str from the same subcycle, so their stress is solved here too.
    That needs their 12 stresses, which therefore evolve identically here
    and on their owner.  G points are local list points with skipU set, so
    this band never updates their velocities;
  - halo slots: every other neighbour of a local list point.  These are
    either list points of other bands or halo slots of the global list.

Stress at a local point reads the velocities of the point and of its ee, ne,
se neighbours from the previous subcycle.  So after every subcycle, the
velocities of G points, and of halo slots that stand for list points of
other bands, are brought from their owners.  Every owned point then sees
exactly the inputs of the single-domain run, and the band's results are
bit-identical to it.

On GPUs the exchange is the library's pack/unpack kernels
(evp1d_exchange_*) around NCCL send/recv, all ordered on the handle's stream.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

STRESS_NB = ("ee", "ne", "se")
STEPU_NB = ("nw", "sw", "sse")
NB = STRESS_NB + STEPU_NB


@dataclass
class Band:
    index: int
    lo: int                 # owned global list points [lo, hi), 0-based
    hi: int
    local: object           # synth.Problem1D of the band
    gid: np.ndarray         # global 0-based position of every local one [local navel]
    sends: dict = field(default_factory=dict)  # peer -> 1-based local list points sent to it
    recvs: dict = field(default_factory=dict)  # peer -> 1-based local positions received from it

    @property
    def n_own(self) -> int:
        return self.hi - self.lo

    def send_idx(self) -> np.ndarray:
        """All sent points in peer order (the layout of the pack buffer)."""
        return _cat([self.sends[q] for q in sorted(self.sends)])

    def recv_idx(self) -> np.ndarray:
        return _cat([self.recvs[q] for q in sorted(self.recvs)])

    def slices(self, which: str) -> dict:
        """peer -> (first, count) of its points in the pack (``"send"``) or
        unpack (``"recv"``) buffer order."""
        d = self.sends if which == "send" else self.recvs
        out, o = {}, 0
        for q in sorted(d):
            out[q] = (o, len(d[q]))
            o += len(d[q])
        return out


def _cat(xs) -> np.ndarray:
    return np.concatenate(xs).astype(np.int32) if xs else np.zeros(0, np.int32)


def bounds(na: int, nbands: int) -> np.ndarray:
    """Band starts [nbands + 1]: equal shares of the list points."""
    if nbands < 1:
        raise ValueError(f"nbands = {nbands} < 1")
    return np.array([(na * b) // nbands for b in range(nbands + 1)], dtype=np.int64)


def split(pr, nbands: int) -> list:
    """Split a Problem1D into `nbands` bands (see the module docstring)."""
    from .synth import Problem1D
    na, navel = pr.na, pr.navel
    starts = bounds(na, nbands)
    nb0 = {k: np.asarray(pr.idx[k], dtype=np.int64) - 1 for k in NB}
    bands = []
    for b in range(nbands):
        lo, hi = int(starts[b]), int(starts[b + 1])
        own = np.arange(lo, hi, dtype=np.int64)
        fwd = np.concatenate([nb0[k][own] for k in STEPU_NB]) if hi > lo else np.zeros(0, np.int64)
        ring = np.unique(fwd[(fwd < na) & ((fwd < lo) | (fwd >= hi))])
        lst = np.concatenate([own, ring])
        nl = len(lst)
        inl = np.zeros(navel, dtype=bool)
        inl[lst] = True
        reach = np.concatenate([nb0[k][lst] for k in NB]) if nl else np.zeros(0, np.int64)
        halo = np.unique(reach[~inl[reach]])
        gid = np.concatenate([lst, halo])
        loc = np.full(navel, -1, dtype=np.int64)
        loc[gid] = np.arange(len(gid))
        idx = {k: (loc[nb0[k][lst]] + 1).astype(np.int32) for k in NB}
        skipU = np.asarray(pr.skipU)[lst].astype(np.int32)
        skipU[hi - lo:] = 1
        local = Problem1D(
            na=nl, navel=len(gid), ndte=pr.ndte, idx=idx,
            skipT=np.asarray(pr.skipT)[lst].astype(np.int32), skipU=skipU,
            f={k: np.ascontiguousarray(v[lst]) for k, v in pr.f.items()},
            stress=np.ascontiguousarray(pr.stress[:, lst]),
            uvel=np.ascontiguousarray(pr.uvel[gid]), vvel=np.ascontiguousarray(pr.vvel[gid]),
            strintx=np.ascontiguousarray(pr.strintx[lst]),
            strinty=np.ascontiguousarray(pr.strinty[lst]),
            Cb=np.ascontiguousarray(pr.Cb[lst]))
        bands.append(Band(index=b, lo=lo, hi=hi, local=local, gid=gid))
    # what each band reads that another band owns: the ring, and halo slots
    # standing for other bands' list points that its stress reads
    for band in bands:
        lp = band.local
        nl = lp.na
        read = np.zeros(lp.navel, dtype=bool)
        read[band.n_own:nl] = True
        for k in STRESS_NB:
            read[np.asarray(lp.idx[k], dtype=np.int64) - 1] = True
        pos = np.nonzero(read & (band.gid < na))[0]
        g = band.gid[pos]
        keep = (g < band.lo) | (g >= band.hi)
        pos, g = pos[keep], g[keep]
        owner = np.searchsorted(starts, g, side="right") - 1
        for q in np.unique(owner):
            sel = owner == q
            order = np.argsort(g[sel], kind="stable")
            band.recvs[int(q)] = (pos[sel][order] + 1).astype(np.int32)
            bands[int(q)].sends[band.index] = (g[sel][order] - bands[int(q)].lo + 1).astype(np.int32)
    return bands


def assemble(pr, bands: list, outs: list) -> dict:
    """Global results from the bands' owned parts.  outs[b] holds the band's
    local arrays (stress [12, na], uvel, vvel [navel], strintx, strinty,
    Cb [na]); halo slots of the global u, v keep the problem's values."""
    res = dict(stress=np.empty_like(pr.stress), uvel=np.array(pr.uvel, dtype=np.float64),
               vvel=np.array(pr.vvel, dtype=np.float64),
               strintx=np.empty(pr.na), strinty=np.empty(pr.na), Cb=np.empty(pr.na))
    for band, o in zip(bands, outs):
        n, lo, hi = band.n_own, band.lo, band.hi
        res["stress"][:, lo:hi] = np.asarray(o["stress"])[:, :n]
        for k in ("uvel", "vvel", "strintx", "strinty", "Cb"):
            res[k][lo:hi] = np.asarray(o[k])[:n]
    return res


def run_band(band: Band, nsub: int, step, pack, unpack, send_buf, recv_buf,
             group=None) -> None:
    """`nsub` subcycles of this rank's band: each is ``step()`` (one subcycle
    of the local solver), ``pack(send_buf)`` (u, v pairs of the sent points),
    point-to-point sends and receives of each peer's slice
    (torch.distributed: NCCL on GPUs, gloo on CPU), then
    ``unpack(recv_buf)``.  The buffers are 1D float64 tensors of 2 x the sent
    and received point counts, on the transport's device."""
    import torch.distributed as dist
    ss, rs = band.slices("send"), band.slices("recv")
    ops = []
    for q, (o, n) in ss.items():
        ops.append(dist.P2POp(dist.isend, send_buf[2 * o: 2 * (o + n)], q, group))
    for q, (o, n) in rs.items():
        ops.append(dist.P2POp(dist.irecv, recv_buf[2 * o: 2 * (o + n)], q, group))
    for _ in range(nsub):
        step()
        pack(send_buf)
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        unpack(recv_buf)


class _DeviceArray:
    """__cuda_array_interface__ of device memory the library owns."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8",
                                         "data": (ptr, False), "version": 3}


def device_view(ptr: int, n: int, device):
    """A float64 torch tensor over `n` doubles of device memory at `ptr`
    (no copy; valid while the owner keeps the memory)."""
    import torch
    if n == 0 or not ptr:
        return torch.zeros(0, dtype=torch.float64, device=device)
    return torch.as_tensor(_DeviceArray(ptr, n), device=device)


class BandSolver:
    """This rank's band on its GPU: an EVP1D handle of the band's local
    problem with the exchange lists set.  The handle's own exchange buffers
    (evp1d_exchange_buffers) are what NCCL sends from and receives into.
    ``run`` mirrors EVP1D.run on the band's local FieldSet; all ranks call
    it together (NCCL point-to-point with the neighbouring bands)."""

    def __init__(self, band: Band, ndte: int = None, params=None, device: int = 0,
                 group=None):
        import torch
        import torch.distributed as dist
        from . import EVP1D
        self.band, self.group = band, group
        self.device = torch.device("cuda", device)
        self.s = EVP1D.from_problem(band.local, ndte=ndte, params=params, device=device)
        self._graphs, self._parity = {}, 0
        self._graph_delta, self.graph_launches = 0, 0
        self.s.exchange_setup(band.send_idx(), band.recv_idx())
        ps, pr = self.s.exchange_buffers()
        self.send_buf = device_view(ps, 2 * len(band.send_idx()), self.device)
        self.recv_buf = device_view(pr, 2 * len(band.recv_idx()), self.device)
        if dist.is_initialized():
            # NCCL creates its communicator on the first collective, which
            # must involve every rank; a band without neighbours posts no
            # point-to-point operation later
            dist.barrier(group=group)

    #: steps per captured CUDA graph (even: a graph leaves the ping-pong
    #: parity where it found it); 0 runs every step eagerly
    GRAPH_STEPS = 50

    def _steps(self, n: int, ends: bool = False) -> None:
        """n band steps; with `ends`, the last one's subcycle ends the call
        (writes strintx, strinty, Cb and str), the others do not."""
        s = self.s
        if n <= 0:
            return
        if ends:
            if n > 1:
                self._steps(n - 1)
            run_band(self.band, 1, lambda: s.subcycles(1), lambda b: s.exchange_pack(),
                     lambda b: s.exchange_unpack(), self.send_buf, self.recv_buf, self.group)
            return
        run_band(self.band, n, lambda: s.subcycles_inner(1), lambda b: s.exchange_pack(),
                 lambda b: s.exchange_unpack(), self.send_buf, self.recv_buf, self.group)

    def subcycles(self, n: int) -> None:
        """`n` subcycles of the uploaded band, each followed by the exchange,
        all ordered on the handle's stream, the last one ending the call.
        Whole chunks of GRAPH_STEPS steps (subcycle, pack, the NCCL
        send/recv, unpack) are captured once per ping-pong parity into a CUDA
        graph and replayed; the rest runs eagerly.  Kernels replayed this way
        are counted in graph_launches."""
        import torch
        s = self.s
        stream = torch.cuda.ExternalStream(s.stream, device=self.device)
        G = self.GRAPH_STEPS
        with torch.cuda.stream(stream):
            # whole graphs, then the rest eagerly, the very last subcycle
            # ending the call
            while G > 0 and n > G and self._graphs is not False:
                g = self._graphs.get(self._parity)
                if g is None:
                    before = s.launch_count()
                    g = torch.cuda.CUDAGraph()
                    try:
                        with torch.cuda.graph(g, stream=stream):
                            self._steps(G)
                    except Exception:
                        # a transport that cannot be captured runs eagerly
                        self._graphs = False
                        break
                    self._graph_delta = s.launch_count() - before
                    self._graphs[self._parity] = g
                g.replay()
                self.graph_launches += self._graph_delta
                n -= G
            self._steps(n, ends=True)
        self._parity ^= n & 1

    def upload(self, fields) -> None:
        self.s.upload(fields)
        self._parity = 0  # the library starts every upload from set 0

    def run(self, ndte: int, fields):
        self.upload(fields)
        self.subcycles(ndte)
        self.s.download(fields)
        return fields

    def finalize(self) -> None:
        # graphs that hold NCCL operations go before the communicator
        self._graphs = {}
        self.s.finalize()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.finalize()
