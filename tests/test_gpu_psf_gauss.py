"""Gaussian PSFs generated on the GPU (psf_gauss, src/psf-gauss.jl:24-55):
spect_psf_gauss_device against the host generator, and a plan built from a
device-generated stack (spect_plan_create_gauss) against the plan built
from the repeated host array (docs/lit/examples/1-overview.jl:91-104).
Tolerance: 1e-6 relative for the PSF values (double precision on both
sides, rounded to float); projections 1e-6 relative."""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ny,px,pz,f0,f1", [(64, 11, 11, 1.0, 3.0), (80, 37, 21, 1.0, 6.0), (16, 7, 1, 0.0, 2.0),
                                            (5, 9, 9, 0.0, 0.0)])
def test_device_generator(S, ny, px, pz, f0, f1):
    import torch

    host = S.psf_gauss(ny=ny, px=px, pz=pz, fwhm_start=f0, fwhm_end=f1)
    dev = torch.empty((ny, pz, px), dtype=torch.float32, device="cuda").permute(2, 1, 0)
    S.psf_gauss_device(dev, ny=ny, px=px, pz=pz, fwhm_start=f0, fwhm_end=f1)
    torch.cuda.synchronize()
    d = dev.cpu().numpy()
    assert d.shape == host.shape
    assert relerr(d, host) <= 1e-6
    # every plane sums to 1 and is point-symmetric
    assert np.allclose(d.sum(axis=(0, 1)), 1.0, atol=1e-5)
    assert np.array_equal(d, d[::-1, ::-1, :])


def test_plan_from_device_psfs(S, O):
    rng = np.random.default_rng(11)
    nx, nz, nview = 64, 40, 24
    mumap = np.asfortranarray(rng.random((nx, nx, nz)) * 0.01, np.float32)
    x = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    psf1 = S.psf_gauss(ny=nx, px=11, pz=11, fwhm_start=1.0, fwhm_end=3.0)
    psfs = np.asfortranarray(np.repeat(psf1[:, :, :, None], nview, axis=3))
    ref = S.SPECTplan(mumap, psfs, 4.8)
    gp = S.SPECTplan.gauss(mumap, 4.8, nview, px=11, fwhm_start=1.0, fwhm_end=3.0)
    assert gp.info()["nset"] == 1
    v0, v1 = S.project(x, ref), S.project(x, gp)
    assert relerr(v1, v0) <= 1e-6
    y = np.asfortranarray(rng.random((nx, nz, nview)), np.float32)
    assert relerr(S.backproject(y, gp), S.backproject(y, ref)) <= 1e-6
    # and against the oracle with the host-generated stack
    G = O.Geometry(mumap, psfs, 4.8)
    assert relerr(v1, G.project(x)) <= 1e-4
    gp.close()
    ref.close()
