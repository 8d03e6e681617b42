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


def test_separable_matches_fft_path(S, O, monkeypatch):
    """Gaussian (rank-1) PSF planes take the direct separable convolution;
    SPECT_CONV=fft forces the FFT kernels.  Both must agree with each other and
    with the oracle (which convolves with the full 2-D kernel)."""
    import importlib

    W = importlib.import_module("spectrecon_b200.workloads")
    st = W.make_study("t", nx=128, nz=80, nview=24, p=37, fwhm_end=6.0, k=6, mu_values=(0.0096, 0.015),
                      nblocks=1, niter=1, seed=3)
    idx = np.array([0, 5, 11, 23], np.int32)
    sep = S.SPECTplan(st.mumap, st.psfs, st.dy)
    monkeypatch.setenv("SPECT_CONV", "fft")
    fft = S.SPECTplan(st.mumap, st.psfs, st.dy)
    monkeypatch.delenv("SPECT_CONV")
    assert sep.conv_kernels() == {"forward": "direct", "adjoint": "direct", "direct_forward_ok": True,
                                  "direct_adjoint_ok": True}
    assert fft.conv_kernels() == {"forward": "fft", "adjoint": "fft", "direct_forward_ok": True,
                                  "direct_adjoint_ok": True}
    v_sep, v_fft = S.project(st.image, sep, index=idx), S.project(st.image, fft, index=idx)
    assert relerr(v_sep, v_fft) <= 1e-5
    G64 = O.Geometry(st.mumap, st.psfs, st.dy, dtype=np.float64)
    assert relerr(v_sep, G64.project(st.image, index=idx)) <= 1e-4
    rng = np.random.default_rng(4)
    y = np.asfortranarray(rng.random((128, 80, idx.size)), np.float32)
    b_sep, b_fft = S.backproject(y, sep, index=idx), S.backproject(y, fft, index=idx)
    assert relerr(b_sep, b_fft) <= 1e-5
    assert relerr(b_sep, G64.backproject(y, index=idx)) <= 1e-4
    sep.close()
    fft.close()


@pytest.mark.gpu
def test_autotune_convolution_choice(S, O):
    """autotune() keeps the faster of the direct and FFT convolution per
    direction; whatever it keeps, results stay within tolerance of the oracle.
    Non-separable PSF planes never get the direct kernels."""
    import importlib

    W = importlib.import_module("spectrecon_b200.workloads")
    st = W.make_study("t", nx=64, nz=48, nview=16, p=17, fwhm_end=4.0, k=4, mu_values=(0.0096, 0.015),
                      nblocks=2, niter=1, seed=5)
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    plan.autotune(8)
    ck = plan.conv_kernels()
    assert ck["direct_forward_ok"] and ck["direct_adjoint_ok"]
    assert ck["forward"] in ("direct", "fft") and ck["adjoint"] in ("direct", "fft")
    G64 = O.Geometry(st.mumap, st.psfs, st.dy, dtype=np.float64)
    idx = np.arange(0, 16, 2, dtype=np.int32)
    assert relerr(S.project(st.image, plan, index=idx), G64.project(st.image, index=idx)) <= 1e-4
    y = np.asfortranarray(np.random.default_rng(6).random((64, 48, idx.size)), np.float32)
    assert relerr(S.backproject(y, plan, index=idx), G64.backproject(y, index=idx)) <= 1e-4
    plan.close()
    # rank-2 planes g1 g2' + g2 g1' (two Gaussian widths) are not separable
    px, pz, ny, nview = st.psfs.shape
    gx1, gx2 = (np.exp(-(np.arange(px) - px // 2) ** 2 / (2 * s * s)) for s in (1.0, 3.0))
    gz1, gz2 = (np.exp(-(np.arange(pz) - pz // 2) ** 2 / (2 * s * s)) for s in (1.0, 3.0))
    plane = np.outer(gx1, gz2) + np.outer(gx2, gz1)
    psfs = np.asfortranarray(np.broadcast_to((plane / plane.sum())[:, :, None, None], (px, pz, ny, nview)),
                             np.float32)
    q = S.SPECTplan(st.mumap, psfs, st.dy)
    assert q.conv_kernels()["forward"] == "fft" and q.conv_kernels()["adjoint"] == "fft"
    q.autotune(8)
    assert q.conv_kernels()["forward"] == "fft" and q.conv_kernels()["adjoint"] == "fft"
    q.close()
