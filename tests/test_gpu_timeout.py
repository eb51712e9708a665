"""The timeout path of the solver's bounded device-side waits, on the GPU.

Every wait of the subcycle kernel is bounded by %globaltimer: the waits on
mbarriers, and the waits of a multi-subcycle launch on the per-tile counters
of the tiles a tile depends on.  One that runs out leaves a code in the
handle's error word, and the next check on the host reports
EVP1D_ERR_TIMEOUT and clears the word.  Here a wait of each kind runs out on
purpose (evp1d_debug_wait_timeout: a barrier that nothing completes;
evp1d_debug_dep_wait_timeout: a counter that nothing raises; a 50 ms limit);
no copy is in flight and nothing faults.  The tests check the reported status
and message, that the word is cleared, and that the same handle then solves
a problem bit for bit like the oracle.
"""
import time

import numpy as np
import pytest

import evp1d
from evp1d import synth, _lib
from test_gpu_parity import assert_same, oracle_run

pytestmark = pytest.mark.gpu


def test_wait_timeout_is_reported_and_the_handle_stays_usable(oracle_mod):
    pr = synth.to_1d(synth.make_grid(60, 40, seed=21, ndte=10))
    ndte = pr.ndte
    with evp1d.EVP1D.from_problem(pr, ndte=ndte) as s:
        s.run(ndte, evp1d.FieldSet.from_problem(pr))
        s.synchronize()  # nothing ran out so far
        t0 = time.perf_counter()
        s.debug_wait_timeout(50_000_000)
        with pytest.raises(evp1d.EVP1DError) as e:
            s.synchronize()
        waited = time.perf_counter() - t0
        assert e.value.code == -5, e.value  # EVP1D_ERR_TIMEOUT
        assert "wait probe" in str(e.value)
        assert 0.04 < waited < 5.0, waited
        s.synchronize()  # the word was cleared
        with pytest.raises(evp1d.EVP1DError) as e:
            s.debug_wait_timeout(10)  # limits outside [1 ms, 1 s] are refused
        assert e.value.code == -1
        fs = evp1d.FieldSet.from_problem(pr)
        s.run(ndte, fs)
    assert_same(fs, oracle_run(oracle_mod, pr, ndte), pr)


def test_dependency_wait_timeout_is_reported_and_the_handle_stays_usable(oracle_mod):
    pr = synth.to_1d(synth.make_grid(60, 40, seed=22, ndte=10))
    ndte = pr.ndte
    with evp1d.EVP1D.from_problem(pr, ndte=ndte) as s:
        s.run(ndte, evp1d.FieldSet.from_problem(pr))
        s.synchronize()
        t0 = time.perf_counter()
        s.debug_dep_wait_timeout(50_000_000)
        with pytest.raises(evp1d.EVP1DError) as e:
            s.synchronize()
        waited = time.perf_counter() - t0
        assert e.value.code == -5, e.value
        assert "dependency-wait probe" in str(e.value)
        assert 0.04 < waited < 5.0, waited
        s.synchronize()
        with pytest.raises(evp1d.EVP1DError) as e:
            s.debug_dep_wait_timeout(10)
        assert e.value.code == -1
        # the probe used a tile counter; the next multi-subcycle call zeroes them
        fs = evp1d.FieldSet.from_problem(pr)
        s.run(ndte, fs)
    assert_same(fs, oracle_run(oracle_mod, pr, ndte), pr)
