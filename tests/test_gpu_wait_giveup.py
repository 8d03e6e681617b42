"""Failure detection of the bounded device waits, without a GPU fault.

The projector kernels wait for bulk copies into shared memory with a bounded
number of mbarrier polls; on give-up a kernel records the failure in a device
flag and returns.  Here a kernel waits on a barrier whose one expected
arrival never happens, so its short wait runs out: the call must come back with
SPECT_ERR_TIMEOUT, the context must stay usable (a projection right after it
matches the oracle), and a plan's flag query reports a clean plan."""
import ctypes

import numpy as np
import pytest

from conftest import relerr, sym_psfs

pytestmark = pytest.mark.gpu

SPECT_OK, SPECT_ERR_TIMEOUT = 0, 16


def test_wait_gives_up_and_context_survives(S, O):
    L = S._native.lib()
    assert L.spect_selftest_wait_timeout() == SPECT_ERR_TIMEOUT
    assert "gave up" in L.spect_last_error().decode()
    rng = np.random.default_rng(3)
    nx, nz, nview = 32, 16, 6
    mumap = np.asfortranarray(0.01 * rng.random((nx, nx, nz)), np.float32)
    psfs = sym_psfs(rng, 5, 3, nx, nview)
    plan = S.SPECTplan(mumap, psfs, 4.8)
    x = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    v = S.project(x, plan)
    assert relerr(v, O.Geometry(mumap, psfs, 4.8).project(x)) <= 1e-4
    assert L.spect_plan_check_error(plan.handle, None) == SPECT_OK
    plan.close()
