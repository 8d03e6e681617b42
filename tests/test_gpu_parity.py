"""GPU parity: the CUDA projector (through the C ABI) against the oracle.

Tolerances: max|gpu - oracle_f32| / max|oracle_f32| <= 1e-4 per projection
set and per reconstruction; adjoint <y, A x> vs <x, A' y> (float64 sums)
<= 1e-5 relative.  Sizes follow the reference's own tests
(test/adjoint-project.jl, test/ml-os-em.jl).
"""
import numpy as np
import pytest

from conftest import relerr, sym_psfs

pytestmark = pytest.mark.gpu

TOL = 1e-4
ADJ_TOL = 1e-5


def _case(rng, nx, nz, nview, px, pz, mu_scale=1.0):
    mumap = np.asfortranarray(mu_scale * rng.random((nx, nx, nz)), np.float32)
    psfs = sym_psfs(rng, px, pz, nx, nview)
    return mumap, psfs


@pytest.mark.parametrize("interp", ["two", "one"])
@pytest.mark.parametrize("nx,nz,nview,px,pz", [(8, 6, 7, 5, 3), (32, 20, 30, 5, 3), (20, 14, 9, 7, 5), (16, 10, 8, 3, 3)])
def test_project_backproject_small(S, O, nx, nz, nview, px, pz, interp):
    """nview = 8 puts views at exact multiples of 90 degrees (the rot_f90-only branch of :one)."""
    rng = np.random.default_rng(nx * 100 + nz)
    mumap, psfs = _case(rng, nx, nz, nview, px, pz, mu_scale=0.02)
    dy = 4.7952
    plan = S.SPECTplan(mumap, psfs, dy, interpmeth=interp)
    G = O.Geometry(mumap, psfs, dy, interp=interp)
    x = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    y = np.asfortranarray(rng.random((nx, nz, nview)), np.float32)
    assert relerr(S.project(x, plan), G.project(x)) <= TOL
    assert relerr(S.backproject(y, plan), G.backproject(y)) <= TOL


@pytest.mark.parametrize("interp", ["two", "one"])
def test_dot_adjoint_32(S, interp):
    """<y, A x> == <x, A' y> (test/adjoint-project.jl:52-106)."""
    rng = np.random.default_rng(52)
    nx, nz, nview = 32, 20, 30
    mumap, psfs = _case(rng, nx, nz, nview, 5, 3)
    plan = S.SPECTplan(mumap, psfs, 4.7952, interpmeth=interp)
    x = np.asfortranarray(rng.standard_normal((nx, nx, nz)), np.float32)
    y = np.asfortranarray(rng.standard_normal((nx, nz, nview)), np.float32)
    a = np.dot(y.ravel().astype(np.float64), S.project(x, plan).ravel().astype(np.float64))
    b = np.dot(x.ravel().astype(np.float64), S.backproject(y, plan).ravel().astype(np.float64))
    assert abs(a - b) <= ADJ_TOL * abs(b)


def test_index_subset(S, O):
    rng = np.random.default_rng(3)
    nx, nz, nview = 16, 10, 12
    mumap, psfs = _case(rng, nx, nz, nview, 5, 5, mu_scale=0.02)
    plan = S.SPECTplan(mumap, psfs, 4.8)
    G = O.Geometry(mumap, psfs, 4.8)
    x = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    idx = np.array([3, 0, 7, 11], np.int32)
    assert relerr(S.project(x, plan, index=idx), G.project(x, index=idx)) <= TOL
    y = np.asfortranarray(rng.random((nx, nz, len(idx))), np.float32)
    assert relerr(S.backproject(y, plan, index=idx), G.backproject(y, index=idx)) <= TOL


def test_osem_mlem(S, O):
    """osem!/mlem! against the oracle (test/ml-os-em.jl:14-53 setup)."""
    rng = np.random.default_rng(14)
    nx, ny, nz, nview = 32, 32, 20, 24
    xtrue = np.zeros((nx, ny, nz), np.float32)
    xtrue[nx // 4:2 * nx // 3, ny // 5:3 * ny // 5, 2 * nz // 6:3 * nz // 6] = 1
    xtrue[2 * nx // 5:3 * nx // 5, ny // 5:2 * ny // 5, 4 * nz // 6:5 * nz // 6] = 2
    xtrue = np.asfortranarray(xtrue)
    psf1 = S.psf_gauss(ny=ny, px=5)
    psfs = np.asfortranarray(np.repeat(psf1[:, :, :, None], nview, axis=3))
    mumap = np.zeros((nx, ny, nz), np.float32, order="F")
    plan = S.SPECTplan(mumap, psfs, 8.0)
    G = O.Geometry(mumap, psfs, 8.0)
    ytrue = G.project(xtrue)
    scale = 20 / ytrue.mean()
    bg = np.full(ytrue.shape, 0.1 * ytrue.mean(), np.float32, order="F")
    yn = np.asfortranarray(rng.poisson(scale * (ytrue + bg)) / scale, np.float32)
    x0 = np.ones((nx, ny, nz), np.float32, order="F")
    assert relerr(S.mlem(x0, yn, bg, plan, niter=3), G.mlem(x0, yn, bg, 3)) <= TOL
    assert relerr(S.osem(x0, yn, bg, S.Ablock(plan, 4), niter=2), G.osem(x0, yn, bg, 4, 2)) <= TOL


@pytest.mark.parametrize("cache", ["0", "1"])
def test_attenuation_cache_on_off(S, O, cache, monkeypatch):
    """Same results with the per-plan attenuation cache on and off."""
    monkeypatch.setenv("SPECT_ATTEN_CACHE", cache)
    rng = np.random.default_rng(77)
    nx, nz, nview = 24, 16, 10
    mumap, psfs = _case(rng, nx, nz, nview, 7, 5, mu_scale=0.03)
    plan = S.SPECTplan(mumap, psfs, 4.8)
    G = O.Geometry(mumap, psfs, 4.8)
    x = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    y = np.asfortranarray(rng.random((nx, nz, nview)), np.float32)
    assert relerr(S.project(x, plan), G.project(x)) <= TOL
    assert relerr(S.backproject(y, plan), G.backproject(y)) <= TOL
