"""The forward projection that allocates nothing (spect_project_static_scratch).

Some callers cannot call cudaMalloc once their plan exists: processes whose
device memory is reserved up front by another allocator (a serving
framework's pool) and real-time pipelines that forbid allocation after
start-up.  For them the library offers spect_project_static_scratch, whose
scratch is one 32 MiB file-scope device array instead of plan buffers.  This
test calls it through the C ABI twice in a row and checks both results
against spect_project, the ordinary entry point, within the parity tolerance
of the other GPU tests; it also checks the rejection of a plan whose single
view needs more scratch than the array holds.  The file name makes pytest
collect it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import relerr, sym_psfs

pytestmark = pytest.mark.gpu

TOL = 1e-4
SPECT_ERR_UNSUPPORTED = 13


def _dev(torch, a):
    """Column-major host array -> device tensor with the same memory order."""
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).cuda()


def test_static_scratch_matches_project(S):
    import torch

    rng = np.random.default_rng(2027)
    nx, nz, nview = 128, 80, 20  # 5.2 MB of rotated planes per view: several groups of views
    mumap = np.asfortranarray(0.01 * rng.random((nx, nx, nz)), np.float32)
    psfs = sym_psfs(rng, 11, 11, nx, nview)
    plan = S.SPECTplan(mumap, psfs, 4.8)
    L = S._native.lib()
    image = _dev(torch, rng.random((nx, nx, nz)))
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    for index in (None, np.array([19, 3, 11, 0, 7, 15, 2], np.int32)):
        n = nview if index is None else len(index)
        ip = None if index is None else index.ctypes.data_as(ctypes.c_void_p)
        ref = torch.empty((n, nz, nx), device="cuda")
        S.check(L.spect_project(plan.handle, ref.data_ptr(), image.data_ptr(), ip, n, sp))
        outs = []
        for _ in range(2):  # two calls in a row share the static array
            out = torch.full((n, nz, nx), float("nan"), device="cuda")
            S.check(L.spect_project_static_scratch(plan.handle, out.data_ptr(), image.data_ptr(), ip, n, sp))
            outs.append(out)
        torch.cuda.synchronize()
        r = ref.cpu().numpy()
        for out in outs:
            o = out.cpu().numpy()
            assert np.isfinite(o).all()
            assert relerr(o, r) <= TOL
    plan.close()


def test_static_scratch_rejects_oversized_plan(S):
    import torch

    rng = np.random.default_rng(5)
    nx, nz, nview = 256, 160, 2  # 42 MB of rotated planes for one view > 32 MiB
    mumap = np.zeros((nx, nx, nz), np.float32, order="F")
    psfs = sym_psfs(rng, 3, 3, nx, nview)
    plan = S.SPECTplan(mumap, psfs, 4.8)
    L = S._native.lib()
    image = torch.zeros((nz, nx, nx), device="cuda")
    out = torch.zeros((nview, nz, nx), device="cuda")
    rc = L.spect_project_static_scratch(plan.handle, out.data_ptr(), image.data_ptr(), None, nview, None)
    assert rc == SPECT_ERR_UNSUPPORTED
    assert "static limit" in L.spect_last_error().decode()
    plan.close()


@pytest.mark.parametrize("case,env", [("one", {}), ("gauss-fused", {}), ("gauss-strip", {"SPECT_ZSTRIP": "1"}),
                                      ("gauss-split-direct", {"SPECT_ZPATH": "0"}),
                                      ("gauss-fft", {"SPECT_CONV": "fft"})])
def test_static_scratch_kernel_paths(S, O, monkeypatch, case, env):
    """Every kernel path through the static array -- the :one shear rotation,
    the fused projector pair (Gaussian, hence separable, PSFs), the
    large-plane pass kernels, the split direct-convolution kernels and the
    FFT kernels -- gives spect_project's result on two calls in a row, and
    the oracle's within the parity tolerance."""
    import torch

    for k, v in env.items():
        monkeypatch.setenv(k, v)
    rng = np.random.default_rng(11)
    nx, nz, nview = 64, 32, 8
    mumap = np.asfortranarray(0.01 * rng.random((nx, nx, nz)), np.float32)
    if case == "one":
        psfs = sym_psfs(rng, 9, 7, nx, nview)
        plan = S.SPECTplan(mumap, psfs, 4.8, interpmeth="one")
    else:
        psfs = np.asfortranarray(np.repeat(S.psf_gauss(ny=nx, px=11, fwhm_start=1, fwhm_end=3)[:, :, :, None],
                                           nview, axis=3))
        plan = S.SPECTplan(mumap, psfs, 4.8)
    assert plan.path == {"gauss-fused": "fused", "gauss-strip": "strip"}.get(case, "split")
    L = S._native.lib()
    x = rng.random((nx, nx, nz)).astype(np.float32)
    image = _dev(torch, x)
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    index = np.array([5, 0, 3, 6], np.int32)
    ip = index.ctypes.data_as(ctypes.c_void_p)
    ref = torch.empty((len(index), nz, nx), device="cuda")
    S.check(L.spect_project(plan.handle, ref.data_ptr(), image.data_ptr(), ip, len(index), sp))
    outs = []
    for _ in range(2):
        out = torch.full((len(index), nz, nx), float("nan"), device="cuda")
        S.check(L.spect_project_static_scratch(plan.handle, out.data_ptr(), image.data_ptr(), ip, len(index), sp))
        outs.append(out)
    torch.cuda.synchronize()
    r = ref.cpu().numpy()
    G = O.Geometry(mumap, psfs, 4.8, interp="one" if case == "one" else "two")
    want = np.ascontiguousarray(G.project(x, index=index).T)  # [view][z][x]
    for out in outs:
        o = out.cpu().numpy()
        assert np.isfinite(o).all()
        assert relerr(o, r) <= TOL
        assert relerr(o, want) <= TOL
    plan.close()
