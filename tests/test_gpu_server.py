"""Serving with continuous batching: results are the same alone and in the mix,
admission respects the device-memory budget, errors come back per job."""
import importlib

import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _studies(O):
    W = importlib.import_module("spectrecon_b200.workloads")
    specs = [dict(nx=32, nz=24, nview=24, p=5, nblocks=4, niter=2),
             dict(nx=48, nz=20, nview=30, p=7, nblocks=5, niter=1),
             dict(nx=64, nz=40, nview=16, p=11, nblocks=8, niter=2)]
    out = []
    for j, sp in enumerate(specs):
        st = W.make_study(f"s{j}", nx=sp["nx"], nz=sp["nz"], nview=sp["nview"], p=sp["p"], fwhm_end=2.0, k=4,
                          mu_values=(0.0096,), nblocks=sp["nblocks"], niter=sp["niter"], seed=700 + j,
                          project_fn=lambda im, s: O.Geometry(s.mumap, s.psfs, s.dy).project(im))
        out.append(st)
    return out


def _submit(srv, st):
    return srv.submit(st.mumap, st.psfs, st.dy, st.ynoisy, st.background, st.nblocks, st.niter)


def test_same_alone_and_in_mix(S, O):
    studies = _studies(O)
    srv = S.Server(max_active=8)
    alone = []
    for st in studies:  # one at a time
        img, lat = srv.wait(_submit(srv, st))
        assert lat > 0
        alone.append(img)
    # the mix: everything at once, the first study twice
    tickets = [_submit(srv, st) for st in studies + [studies[0]]]
    mixed = [srv.wait(t)[0] for t in tickets]
    for k, st in enumerate(studies + [studies[0]]):
        ref = alone[k % len(studies)]
        assert relerr(mixed[k], ref) <= TOL
    st = studies[2]
    x0 = np.ones(st.image.shape, np.float32, order="F")
    ref_cpu = O.Geometry(st.mumap, st.psfs, st.dy).osem(x0, st.ynoisy, st.background, st.nblocks, st.niter)
    assert relerr(alone[2], ref_cpu) <= TOL
    stats = srv.stats()
    assert stats["done"] == 7 and stats["failed"] == 0 and stats["max_active_seen"] >= 2
    srv.close()


def test_admission_by_memory_budget(S, O):
    studies = _studies(O)
    # a budget that holds one small job at a time: the others wait and run later
    srv = S.Server(budget_bytes=30 << 20, max_active=8)
    tickets = [_submit(srv, studies[0]) for _ in range(3)]
    res = [srv.wait(t)[0] for t in tickets]
    for r in res[1:]:
        assert relerr(r, res[0]) <= TOL
    stats = srv.stats()
    assert stats["done"] == 3 and stats["max_active_seen"] == 1
    srv.close()


def test_errors_per_job(S, O):
    st = _studies(O)[0]
    srv = S.Server(budget_bytes=1 << 20, max_active=2)  # 1 MiB: too small for any job
    with pytest.raises(S.SpectError) as e:
        srv.submit(st.mumap, st.psfs, st.dy, st.ynoisy, st.background, 5, 1)
    assert str(e.value) == "nview must be divisible by nblocks!"
    with pytest.raises(S.SpectError) as e:
        srv.submit(st.mumap, st.psfs, st.dy, st.ynoisy, np.zeros_like(st.background), 4, 1)
    assert str(e.value) == "need background > 0"
    t = _submit(srv, st)
    with pytest.raises(S.SpectError) as e:
        srv.wait(t)
    assert "above the server budget" in str(e.value)
    srv.close()
