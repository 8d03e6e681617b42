"""2-D (nz = 1, pz = 1) and axial-blur-free (pz = 1) geometries, and the
GPU-resident operator with custom-Jacobian autograd.

2-D follows docs/lit/examples/5-2d.jl (a 3-D array with nz = 1 and PSFs of
support px x 1); the operator follows the LinearMapAA closures of Ablock
(src/ml-os-em.jl:70-84) and the custom adjoints of
docs/lit/examples/6-dl.jl:152-156.  Tolerance: max|gpu - oracle| / max|oracle|
<= 1e-4 against the float32 and the float64 oracle; adjoint dot test <= 1e-5.
"""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _geometry(S, rng, nx, nz, px, pz, nview, fwhm_end):
    mumap = np.zeros((nx, nx, nz), np.float32)
    c = (nx - 1) / 2
    xx, yy = np.meshgrid(np.arange(nx) - c, np.arange(nx) - c, indexing="ij")
    mumap[(xx / (0.42 * nx)) ** 2 + (yy / (0.36 * nx)) ** 2 <= 1] = 0.0096
    mumap = np.asfortranarray(mumap)
    psf1 = S.psf_gauss(ny=nx, px=px, pz=pz, fwhm_start=1, fwhm_end=fwhm_end)
    psfs = np.asfortranarray(np.repeat(psf1[:, :, :, None], nview, axis=3), np.float32)
    x = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    return mumap, psfs, x


@pytest.mark.parametrize("nx,nz,px,pz,nview,idx", [
    (128, 1, 11, 1, 80, [0, 13, 40, 79]),   # the 2-D example: 128x128x1, 11x1 PSF, 80 views
    (64, 1, 7, 1, 32, None),                # 2-D, all views
    (64, 40, 11, 1, 24, [1, 12, 23]),       # 3-D volume, no axial blur
    (64, 3, 9, 3, 16, [0, 5]),              # thin slab: padded plane 128x8
])
def test_thin_geometries(S, O, nx, nz, px, pz, nview, idx):
    rng = np.random.default_rng(nx + nz + px + pz)
    mumap, psfs, x = _geometry(S, rng, nx, nz, px, pz, nview, 3.0)
    plan = S.SPECTplan(mumap, psfs, 4.8)
    G32 = O.Geometry(mumap, psfs, 4.8)
    G64 = O.Geometry(mumap, psfs, 4.8, dtype=np.float64)
    ii = None if idx is None else np.array(idx, np.int32)
    v = S.project(x, plan, index=ii)
    assert relerr(v, G32.project(x, index=ii)) <= TOL
    assert relerr(v, G64.project(x, index=ii)) <= TOL
    n = nview if ii is None else ii.size
    y = np.asfortranarray(rng.random((nx, nz, n)), np.float32)
    b = S.backproject(y, plan, index=ii)
    assert relerr(b, G32.backproject(y, index=ii)) <= TOL
    assert relerr(b, G64.backproject(y, index=ii)) <= TOL
    lhs = float(np.dot(np.ravel(v, order="F").astype(np.float64), np.ravel(y, order="F").astype(np.float64)))
    rhs = float(np.dot(np.ravel(x, order="F").astype(np.float64), np.ravel(b, order="F").astype(np.float64)))
    assert abs(lhs - rhs) <= 1e-5 * abs(rhs)


def test_2d_mlem(S, O):
    """ML-EM on the 2-D geometry (docs/lit/examples/5-2d.jl runs mlem!)."""
    rng = np.random.default_rng(52)
    mumap, psfs, x = _geometry(S, rng, 64, 1, 11, 1, 32, 3.0)
    plan = S.SPECTplan(mumap, psfs, 4.8)
    G = O.Geometry(mumap, psfs, 4.8)
    ytrue = G.project(x)
    bg = np.full(ytrue.shape, 0.05 * ytrue.mean(), np.float32, order="F")
    y = np.asfortranarray(rng.poisson(ytrue + bg).astype(np.float32))
    x0 = np.ones(x.shape, np.float32, order="F")
    a = S.mlem(x0, y, bg, plan, niter=3)
    assert relerr(a, G.osem(x0, y, bg, 1, 3)) <= TOL


def test_operator_and_autograd(S, O):
    import torch
    import importlib

    op = importlib.import_module("spectrecon_b200.operator")
    rng = np.random.default_rng(7)
    mumap, psfs, x = _geometry(S, rng, 64, 24, 11, 11, 30, 3.0)
    plan = S.SPECTplan(mumap, psfs, 4.8)
    G = O.Geometry(mumap, psfs, 4.8)
    idx = np.arange(2, 30, 5, dtype=np.int32)
    A = op.SPECTOperator(plan, idx)
    assert A.shape == (64 * 24 * idx.size, 64 * 64 * 24) and A.T.shape == A.shape[::-1]
    xt = torch.from_numpy(np.ascontiguousarray(x.transpose(2, 1, 0))).cuda().permute(2, 1, 0)
    yt = A @ xt
    assert tuple(yt.shape) == (64, 24, idx.size)
    assert relerr(yt.cpu().numpy(), G.project(x, index=idx)) <= TOL
    # custom Jacobian: d/dx <w, A x> = A' w, and d/dy <u, A' y> = A u
    w = torch.rand(yt.shape, device="cuda", dtype=torch.float32)
    xg = xt.clone().requires_grad_(True)
    (op.project_ad(xg, A) * w).sum().backward()
    ref = G.backproject(np.asfortranarray(w.cpu().numpy()), index=idx)
    assert relerr(xg.grad.cpu().numpy(), ref) <= TOL
    yg = w.clone().requires_grad_(True)
    (op.backproject_ad(yg, A) * xt).sum().backward()
    assert relerr(yg.grad.cpu().numpy(), G.project(x, index=idx)) <= TOL
    # row-major torch tensors are accepted (copied into the column-major layout)
    yt2 = A @ xt.contiguous()
    assert torch.equal(yt2, yt)
