"""GPU parity at the benchmark workloads' padded sizes (C ABI vs oracle).

Covers every code path of the convolution kernels: register accumulators
(256x128, 128x128 padded planes), global accumulator slabs (256x256,
512x256), and B in global memory (512x512).  Views are subsampled where the
oracle would otherwise take minutes; the per-view arithmetic is identical.
Tolerance: max|gpu - oracle_f32| / max|oracle_f32| <= 1e-4; the error against
the float64 oracle is asserted at the same bound.
"""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-4

def _study(S, nx, nz, nview, p, fwhm_end, mu_values, seed):
    import importlib
    W = importlib.import_module("spectrecon_b200.workloads")
    return W.make_study("t", nx=nx, nz=nz, nview=nview, p=p, fwhm_end=fwhm_end, k=6, mu_values=mu_values,
                        nblocks=1, niter=1, seed=seed)

@pytest.mark.parametrize("nx,nz,nview,p,fwhm,idx", [
    (64, 64, 64, 11, 3.0, [0, 5, 16, 31, 47]),            # 64x64x64, 11x11 PSF: 128x128 padded
    (128, 80, 120, 37, 6.0, [0, 7, 30, 61, 119]),          # 128x128x80, 37x37 PSF: 256x128 padded
    (128, 128, 60, 37, 6.0, [3, 29]),                      # 128x128x128, 37x37 PSF: 256x256 padded (global slabs)
    (96, 48, 90, 21, 3.5, [0, 44, 89]),                    # 96x96x48, 21x21 PSF: 128x128 padded
])
def test_config_parity(S, O, nx, nz, nview, p, fwhm, idx):
    st = _study(S, nx, nz, nview, p, fwhm, (0.0096, 0.015), seed=nx + nz + p)
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    G32 = O.Geometry(st.mumap, st.psfs, st.dy)
    G64 = O.Geometry(st.mumap, st.psfs, st.dy, dtype=np.float64)
    idx = np.array(idx, np.int32)
    v = S.project(st.image, plan, index=idx)
    assert relerr(v, G32.project(st.image, index=idx)) <= TOL
    assert relerr(v, G64.project(st.image, index=idx)) <= TOL
    rng = np.random.default_rng(1)
    y = np.asfortranarray(rng.random((nx, nz, len(idx))), np.float32)
    b = S.backproject(y, plan, index=idx)
    assert relerr(b, G32.backproject(y, index=idx)) <= TOL
    assert relerr(b, G64.backproject(y, index=idx)) <= TOL

@pytest.mark.parametrize("path", ["strip", "split"])
def test_large_512_planes(S, O, monkeypatch, path):
    """Largest plane: 256x256x200 image, 65x65 PSF -> 512x512 padded planes,
    through the large-plane pass kernels (the default here) and through the
    split kernels (SPECT_ZSTRIP=0: FFT convolution, B in global memory).

    At this size the reference's own Float32 adjoint carries ~1.8e-4 of FFT
    round-off (fft_conv_adj! sums all 128+156 padded rows/columns into the edge
    pixels, src/fft_convolve.jl:100-122), so the GPU result is held to 1e-4
    against the Float64 oracle and to the oracle's own f32-vs-f64 error
    against the Float32 oracle."""
    monkeypatch.setenv("SPECT_ZSTRIP", "1" if path == "strip" else "0")
    st = _study(S, 256, 200, 128, 65, 10.0, (0.0096, 0.015, 0.004), seed=5)
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    assert plan.path == path
    G = O.Geometry(st.mumap, st.psfs, st.dy)
    G64 = O.Geometry(st.mumap, st.psfs, st.dy, dtype=np.float64)
    idx = np.array([17], np.int32)
    v64 = G64.project(st.image, index=idx)
    v = S.project(st.image, plan, index=idx)
    assert relerr(v, G.project(st.image, index=idx)) <= TOL
    assert relerr(v, v64) <= TOL
    rng = np.random.default_rng(2)
    y = np.asfortranarray(rng.random((256, 200, 1)), np.float32)
    b = S.backproject(y, plan, index=idx)
    b32, b64 = G.backproject(y, index=idx), G64.backproject(y, index=idx)
    assert relerr(b, b64) <= TOL
    assert relerr(b, b32) <= max(TOL, 1.5 * relerr(b32, b64))

def test_full_128x128x80_subset_osem_update(S, O):
    """One OS-EM iteration (8 subsets of 15 views) of the benchmark study vs the oracle."""
    import importlib
    W = importlib.import_module("spectrecon_b200.workloads")
    st = W.named_study("larger_128x128x80", project_fn=lambda im, s: O.Geometry(s.mumap, s.psfs, s.dy).project(im))
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    G = O.Geometry(st.mumap, st.psfs, st.dy)
    x0 = np.ones(st.image.shape, np.float32, order="F")
    a = S.osem(x0, st.ynoisy, st.background, S.Ablock(plan, 8), niter=1)

    b = G.osem(x0, st.ynoisy, st.background, 8, 1)
    assert relerr(a, b) <= TOL


def test_config_parity_one(S, O):
    """interpmeth :one at the single larger study's sizes (256x128 padded planes, L = 184)."""
    st = _study(S, 128, 80, 120, 37, 6.0, (0.0096, 0.015), seed=9)
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy, interpmeth="one")
    G = O.Geometry(st.mumap, st.psfs, st.dy, interp="one")
    idx = np.array([0, 30, 45, 77], np.int32)  # includes 90 degrees (view 30 of 120)
    assert relerr(S.project(st.image, plan, index=idx), G.project(st.image, index=idx)) <= TOL
    rng = np.random.default_rng(3)
    y = np.asfortranarray(rng.random((128, 80, len(idx))), np.float32)
    assert relerr(S.backproject(y, plan, index=idx), G.backproject(y, index=idx)) <= TOL


@pytest.mark.parametrize("nbuf,zw,stages", [("1", "8", "1"), ("2", "8", "2"), ("1", "16", "2"), ("2", "16", "1")])
def test_fused_pair_plane_walk(S, O, monkeypatch, nbuf, zw, stages):
    """Fused pair walking several work items per block (60 views of 64x64x40:
    more (view, depth chunk) items than SMs), convolution tasks of 8 and of 16
    outputs, the adjoint x pass with one and with two buffers, the forward
    with one and with two staging buffers; all views, a subset, and one OS-EM
    iteration."""
    monkeypatch.setenv("SPECT_ZADJ_BUFFERS", nbuf)
    monkeypatch.setenv("SPECT_ZW", zw)
    monkeypatch.setenv("SPECT_ZFWD_STAGES", stages)
    st = _study(S, 64, 40, 60, 11, 3.0, (0.0096, 0.015), seed=5)
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    assert plan.fused
    G = O.Geometry(st.mumap, st.psfs, st.dy)
    assert relerr(S.project(st.image, plan), G.project(st.image)) <= TOL
    rng = np.random.default_rng(4)
    y = np.asfortranarray(rng.random((64, 40, 60)), np.float32)
    assert relerr(S.backproject(y, plan), G.backproject(y)) <= TOL
    idx = np.array([1, 13, 44], np.int32)
    ys = np.asfortranarray(y[:, :, idx])
    assert relerr(S.backproject(ys, plan, index=idx), G.backproject(ys, index=idx)) <= TOL
    x0 = np.ones(st.image.shape, np.float32, order="F")
    yn = np.asfortranarray(np.maximum(G.project(st.image), 0) + 1, np.float32)
    bg = np.full(yn.shape, 1.0, np.float32, order="F")
    assert relerr(S.osem(x0, yn, bg, S.Ablock(plan, 4), niter=1), G.osem(x0, yn, bg, 4, 1)) <= TOL


def test_fused_pair_odd_width(S, O):
    """Fused pair with nx = 40 (a multiple of 8, not of 16: 8-output tasks)
    and nz = 37 (a partial last z task)."""
    st = _study(S, 40, 37, 24, 9, 2.5, (0.0096, 0.015), seed=11)
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    assert plan.fused
    G = O.Geometry(st.mumap, st.psfs, st.dy)
    assert relerr(S.project(st.image, plan), G.project(st.image)) <= TOL
    rng = np.random.default_rng(6)
    y = np.asfortranarray(rng.random((40, 37, 24)), np.float32)
    assert relerr(S.backproject(y, plan), G.backproject(y)) <= TOL


def test_trimmed_taps_match_full(S, O, monkeypatch):
    """Skipping the outer PSF taps below Float32 resolution (the default)
    against every tap (SPECT_ZTRIM=0): the same projections and
    back-projections to 1e-6, both within the oracle tolerance."""
    st = _study(S, 128, 80, 120, 37, 6.0, (0.0096, 0.015), seed=21)
    idx = np.array([0, 7, 30, 61, 119], np.int32)
    rng = np.random.default_rng(8)
    y = np.asfortranarray(rng.random((128, 80, len(idx))), np.float32)
    out = {}
    for trim in ("1", "0"):
        monkeypatch.setenv("SPECT_ZTRIM", trim)
        plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
        assert plan.fused
        out[trim] = (S.project(st.image, plan, index=idx), S.backproject(y, plan, index=idx))
    G = O.Geometry(st.mumap, st.psfs, st.dy)
    v_ref, b_ref = G.project(st.image, index=idx), G.backproject(y, index=idx)
    for trim in ("1", "0"):
        assert relerr(out[trim][0], v_ref) <= TOL
        assert relerr(out[trim][1], b_ref) <= TOL
    assert relerr(out["1"][0], out["0"][0]) <= 1e-6
    assert relerr(out["1"][1], out["0"][1]) <= 1e-6


def test_wide_psf_takes_split_path(S, O):
    """A PSF row longer than the fused passes' 9 blocks of 8 taps (75 taps)
    runs the split kernels, with the same results as the oracle."""
    st = _study(S, 64, 24, 12, 75, 6.0, (0.0096, 0.015), seed=31)
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    assert not plan.fused
    G = O.Geometry(st.mumap, st.psfs, st.dy)
    idx = np.array([0, 5], np.int32)
    assert relerr(S.project(st.image, plan, index=idx), G.project(st.image, index=idx)) <= TOL


def test_large_plane_kernels_match_fused_bitwise(S, O, monkeypatch):
    """The large-plane kernels (one kernel per pass over plane tiles) run every
    output through the fused kernels' operations in the same order: forced on
    the single larger study's geometry they give the fused pair's projections,
    back-projections and OS-EM iterate bit for bit."""
    st = _study(S, 128, 80, 120, 37, 6.0, (0.0096, 0.015), seed=41)
    idx = np.array([0, 7, 30, 61, 119], np.int32)
    rng = np.random.default_rng(9)
    y = np.asfortranarray(rng.random((128, 80, len(idx))), np.float32)
    x0 = np.ones(st.image.shape, np.float32, order="F")
    yn = np.asfortranarray(rng.random((128, 80, 120)) + 0.5, np.float32)
    bg = np.full(yn.shape, 0.1, np.float32, order="F")
    out = {}
    for strip in ("0", "1"):
        monkeypatch.setenv("SPECT_ZSTRIP", strip)
        plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
        assert plan.path == ("strip" if strip == "1" else "fused")
        out[strip] = (S.project(st.image, plan, index=idx), S.backproject(y, plan, index=idx),
                      S.osem(x0, yn, bg, S.Ablock(plan, 8), niter=1))
    for a, b in zip(out["0"], out["1"]):
        assert np.array_equal(a, b)
    G = O.Geometry(st.mumap, st.psfs, st.dy)
    assert relerr(out["1"][0], G.project(st.image, index=idx)) <= TOL
