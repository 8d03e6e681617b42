"""The arithmetic of the direct separable convolution kernels (csrc/sconv.cuh),
restated in numpy and checked against the oracle's FFT convolution
(fft_conv!/fft_conv_adj!, src/fft_convolve.jl:33-130) on the CPU.

For a rank-1 plane h[d, e] = a[d] b[e] the kernels compute
  forward: a z pass then an x pass, each over a line whose out-of-range
           samples are clamped (replicated) -- taps read as w[m] = factor[p-1-m]
           over the padded line;
  adjoint: zero-padded correlations with the factors plus, at the two ends
           of each line, the folded padding as dot products with the tail
           sums cL_k = sum_{d>k} w(d), cR_k = sum_{d<-k} w(d).
Both must equal the oracle's replicate-boundary convolution and its adjoint
(tolerance 1e-12 relative in float64), also when the kernel is wider than
the image (h >= n), where the tails reach into the zero padding."""
import numpy as np
import pytest

from conftest import relerr


def gauss(p, sigma):
    x = np.arange(p) - (p - 1) // 2
    g = np.exp(-x * x / (2.0 * sigma * sigma))
    return g / g.sum()


def clamp_pass(line, w):
    """out[i] = sum_m w[m] line[clamp(i + m - h)], w = reversed factor."""
    n, p = line.shape[0], w.shape[0]
    h = (p - 1) // 2
    idx = np.clip(np.arange(n)[:, None] + np.arange(p)[None, :] - h, 0, n - 1)
    return np.tensordot(line[idx], w, axes=([1], [0]))


def tails(w):
    h = (w.shape[0] - 1) // 2
    cl = np.array([w[h + k + 1:].sum() for k in range(h)])
    cr = np.array([w[:h - k].sum() for k in range(h)])
    return cl, cr


def corr_adj_pass(u, w):
    """Transpose of clamp_pass along axis 0: zero-padded correlation plus the
    folded padding at both ends."""
    n, p = u.shape[0], w.shape[0]
    h = (p - 1) // 2
    pad = np.zeros((n + 2 * h,) + u.shape[1:])
    pad[h:h + n] = u
    out = sum(w[m] * pad[m:m + n] for m in range(p))
    cl, cr = tails(w)
    for k in range(h):
        if k < n:
            out[0] = out[0] + cl[k] * u[k]
            out[n - 1] = out[n - 1] + cr[k] * u[n - 1 - k]
    return out


def sep_forward(img, a, b):
    bz = clamp_pass(img.T, b[::-1]).T          # z pass (axis 1)
    return clamp_pass(bz, a[::-1])              # x pass (axis 0)


def sep_adjoint(v, a, b):
    wx = corr_adj_pass(v, a)                    # x pass first (transpose order)
    return corr_adj_pass(wx.T, b).T             # then z


CASES = [(16, 12, 5, 7, 1.0, 2.0), (32, 20, 11, 9, 2.5, 1.5), (8, 6, 21, 15, 4.0, 3.0),
         (24, 1, 7, 1, 1.2, 1.0), (16, 3, 9, 9, 2.0, 2.0)]


@pytest.mark.parametrize("nx,nz,px,pz,sx,sz", CASES)
def test_direct_forward_equals_fft_conv(O, nx, nz, px, pz, sx, sz):
    rng = np.random.default_rng(nx * 100 + px)
    img = rng.random((nx, nz))
    a, b = gauss(px, sx), gauss(pz, sz)
    ref = O.fft_conv(img, np.outer(a, b), dtype=np.float64)
    assert relerr(sep_forward(img, a, b), ref) <= 1e-12


@pytest.mark.parametrize("nx,nz,px,pz,sx,sz", CASES)
def test_direct_adjoint_equals_fft_conv_adj(O, nx, nz, px, pz, sx, sz):
    rng = np.random.default_rng(nx * 100 + pz)
    v = rng.random((nx, nz))
    a, b = gauss(px, sx), gauss(pz, sz)
    ref = O.fft_conv(v, np.outer(a, b), adj=True, dtype=np.float64)
    assert relerr(sep_adjoint(v, a, b), ref) <= 1e-12


@pytest.mark.parametrize("nx,nz,px,pz,sx,sz", CASES[:3])
def test_direct_pair_is_adjoint(nx, nz, px, pz, sx, sz):
    """<A x, y> == <x, A' y> for the restated direct pair itself."""
    rng = np.random.default_rng(7 + nx)
    x, y = rng.random((nx, nz)), rng.random((nx, nz))
    a, b = gauss(px, sx), gauss(pz, sz)
    lhs = np.vdot(sep_forward(x, a, b), y)
    rhs = np.vdot(x, sep_adjoint(y, a, b))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
