"""Failures made on the host, and the solver's state after every subcycle.

- Allocation failures (evp1d_debug_fail_alloc).  The reference stops the
  program on a failed allocation (integration/ice_dyn_evp1d.F90:394-460);
  the library must return EVP1D_ERR_NOMEM instead, free what the call had
  allocated, and leave the handle usable.  Each device allocation site is
  made to fail once: the handle's arena (evp1d_init), the exchange lists,
  the autotuner's backup, the adjoint's work arrays and checkpoint store,
  and the 2D adapter's buffers.  Nothing faults on the GPU: the failing
  allocation is never attempted.
- The state after every subcycle, not only at the end of a call, equals
  the oracle's, with a scan for non-finite outputs.
"""
import numpy as np
import pytest
import torch

import evp1d
from evp1d import synth
from test_gpu_parity import assert_same, oracle_run

pytestmark = pytest.mark.gpu

NOMEM = -4


@pytest.fixture(autouse=True)
def _disarm():
    yield
    evp1d.debug_fail_alloc(0)


def _nomem(fn):
    with pytest.raises(evp1d.EVP1DError) as e:
        fn()
    assert e.value.code == NOMEM, e.value
    return e.value


def test_failed_device_allocations(oracle_mod):
    pr = synth.to_1d(synth.make_grid(60, 40, seed=5, ndte=6, curvilinear=True))
    ref = oracle_run(oracle_mod, pr, 6)
    u_obs, v_obs = synth.observations(pr.na, 99)

    def grads(s):
        fs = evp1d.FieldSet.from_problem(pr)
        s.run_checkpointed(6, fs, interval=3)
        return s.adjoint(2 * (fs.uvel[: pr.na] - u_obs), 2 * (fs.vvel[: pr.na] - v_obs))

    with evp1d.EVP1D.from_problem(pr, ndte=6) as s:
        g_ref = grads(s)

    evp1d.debug_fail_alloc(1)
    err = _nomem(lambda: evp1d.EVP1D.from_problem(pr, ndte=6))
    assert "alloc" in str(err).lower() or "memory" in str(err).lower(), err
    with evp1d.EVP1D.from_problem(pr, ndte=6) as s:  # the injection fired once
        fs = evp1d.FieldSet.from_problem(pr)
        s.upload(fs)
        evp1d.debug_fail_alloc(1)
        _nomem(lambda: s.exchange_setup([1, 2], [pr.na + 1]))
        evp1d.debug_fail_alloc(1)
        _nomem(lambda: s.autotune(2))
        for n in (1, 2):  # the adjoint's work arrays, then its checkpoint store
            evp1d.debug_fail_alloc(n)
            _nomem(lambda: grads(s))
        evp1d.debug_fail_alloc(0)
        fs = evp1d.FieldSet.from_problem(pr)
        s.run(6, fs)
        assert_same(fs, ref, pr)
        g = grads(s)
        for k in g_ref:
            assert np.array_equal(np.asarray(g[k]).view(np.int64),
                                  np.asarray(g_ref[k]).view(np.int64)), k
        s.exchange_setup([1, 2], [pr.na + 1])

    from evp1d import dyn
    gr = synth.make_grid(40, 30, seed=7, ndte=4)
    p = evp1d.set_evp_parameters(4)
    for n in (1, 2, 3):  # the solver's arena, then the adapter's cell map and 2D fields
        evp1d.debug_fail_alloc(n)
        _nomem(lambda: dyn.Dyn2D(gr.tmask, gr.f["dyT"], gr.f["dxT"], gr.f["uarear"],
                                 gr.f["HTE"], gr.f["HTN"], p))
    evp1d.debug_fail_alloc(0)
    with dyn.Dyn2D(gr.tmask, gr.f["dyT"], gr.f["dxT"], gr.f["uarear"], gr.f["HTE"],
                   gr.f["HTN"], p) as d:
        d.run(4, dyn.fields_from_grid(gr), gr.iceT, gr.iceU)


def test_failed_allocations_free_what_they_took():
    """Failures after earlier allocations of the same call (the 2D adapter:
    the solver's arena and the cell map are taken when its 2D fields fail),
    repeated on a 300 x 200 grid (tens of MB each): free device memory comes
    back to where it was."""
    from evp1d import dyn
    gr = synth.make_grid(300, 200, seed=8, ndte=2)
    p = evp1d.set_evp_parameters(2)
    args = (gr.tmask, gr.f["dyT"], gr.f["dxT"], gr.f["uarear"], gr.f["HTE"], gr.f["HTN"], p)
    with dyn.Dyn2D(*args) as d:  # modules loaded, pools settled
        d.run(2, dyn.fields_from_grid(gr), gr.iceT, gr.iceU)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        for n in (2, 3):
            evp1d.debug_fail_alloc(n)
            _nomem(lambda: dyn.Dyn2D(*args))
    evp1d.debug_fail_alloc(0)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 >= free0 - (8 << 20), (free0, free1)


def test_every_subcycle_matches_the_oracle(oracle_mod):
    """One subcycle per call on the device-resident state, downloaded and
    compared with the oracle advanced by one subcycle (the same ndte
    parameters) after each; no output is NaN or infinite."""
    ndte = 8
    pr = synth.to_1d(synth.make_grid(70, 50, seed=31, ndte=ndte, curvilinear=True))
    p = oracle_mod.params(ndte)
    op = oracle_mod.OracleParams(**{k: getattr(p, k) for k in evp1d._lib.PARAM_FIELDS})
    st = oracle_mod.State1D(pr)
    fs = evp1d.FieldSet.from_problem(pr)
    with evp1d.EVP1D.from_problem(pr, ndte=ndte) as s:
        s.upload(fs)
        for _ in range(ndte):
            s.subcycles(1)
            s.download(fs)
            oracle_mod.run_1d(pr, 1, p=op, state=st)
            assert_same(fs, st, pr)
            for a in (fs.stress, fs.uvel, fs.vvel, fs.strintx, fs.strinty, fs.Cb):
                assert np.all(np.isfinite(a))
