"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline /
``--impl reference`` arm may import this module; it is the checker, never the
product path.  Arrays use the reference's Julia (column-major) layout, i.e.
numpy arrays indexed like Julia, ``image[x,y,z]`` of shape ``(nx, ny, nz)``,
``views`` ``(nx, nz, nview)``, ``psfs`` ``(px, pz, ny, nview)``, stored
column-major (``order='F'``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> str:
    """Compile liboracle.so with the committed Makefile (no-op when fresh)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "spect_oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        _LIB = ctypes.CDLL(path)
        _declare(_LIB)
    return _LIB


_P = ctypes.c_void_p
_I = ctypes.c_int


def _declare(L):
    for sfx, T in (("f32", ctypes.c_float), ("f64", ctypes.c_double)):
        getattr(L, f"oracle_project_{sfx}").argtypes = [_P, _P, _P, _P, _I, _I, _I, _I, _I, T, _I, _P, _P, _I, _I]
        getattr(L, f"oracle_backproject_{sfx}").argtypes = [_P, _P, _P, _P, _I, _I, _I, _I, _I, T, _I, _P, _P, _I, _I]
        getattr(L, f"oracle_mlem_{sfx}").argtypes = [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, T, _I, _P, _I, _I]
        getattr(L, f"oracle_osem_{sfx}").argtypes = [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, T, _I, _P, _I, _I, _I]
        getattr(L, f"oracle_imrotate_{sfx}").argtypes = [_P, _P, _I, T, _I, _I]
        getattr(L, f"oracle_fft_conv_{sfx}").argtypes = [_P, _P, _I, _I, _P, _I, _I, _I]
        getattr(L, f"oracle_rot_f90_{sfx}").argtypes = [_P, _P, _I, _I, _I]
        getattr(L, f"oracle_default_angle_{sfx}").argtypes = [_I, _I]
        getattr(L, f"oracle_default_angle_{sfx}").restype = T
    for name in ("oracle_padzero_f32", "oracle_padrepl_f32"):
        getattr(L, name).argtypes = [_P, _P, _I, _I, _I, _I, _I, _I]
    L.oracle_pad2sizezero_f32.argtypes = [_P, _P, _I, _I, _I, _I]
    L.oracle_fftshift2_f32.argtypes = [_P, _P, _I, _I]
    L.oracle_rot_padsize.argtypes = [_I]
    L.oracle_power2.argtypes = [_I]


def _dt(dtype):
    dtype = np.dtype(dtype)
    if dtype == np.float32:
        return "f32", np.float32
    if dtype == np.float64:
        return "f64", np.float64
    raise TypeError(f"oracle supports float32/float64, got {dtype}")


def _c(a, dt):
    return np.asfortranarray(a, dtype=dt)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _nthread(n):
    return int(n) if n else (os.cpu_count() or 1)


class Geometry:
    """Sizes and fixed inputs of one system model (mirrors SPECTplan's data)."""

    def __init__(self, mumap, psfs, dy, interp="two", viewangle=None, dtype=np.float32, nthread=None):
        self.sfx, self.dt = _dt(dtype)
        self.mumap = _c(mumap, self.dt)
        self.psfs = _c(psfs, self.dt)
        self.nx, self.ny, self.nz = self.mumap.shape
        self.px, self.pz, ny2, self.nview = self.psfs.shape
        assert ny2 == self.ny
        self.dy = float(dy)
        self.interp = 1 if interp in ("one", 1, ":one") else 2
        self.angles = None if viewangle is None else np.ascontiguousarray(viewangle, dtype=self.dt)
        self.nthread = _nthread(nthread)

    def _args(self):
        return (self.nx, self.nz, self.px, self.pz, self.nview, self.dy, self.interp, _ptr(self.angles))

    def project(self, image, index=None):
        image = _c(image, self.dt)
        idx = None if index is None else np.ascontiguousarray(index, dtype=np.int32)
        n = self.nview if idx is None else len(idx)
        views = np.empty((self.nx, self.nz, n), dtype=self.dt, order="F")
        fn = getattr(lib(), f"oracle_project_{self.sfx}")
        rc = fn(_ptr(views), _ptr(image), _ptr(self.mumap), _ptr(self.psfs), *self._args(),
                _ptr(idx), n, self.nthread)
        assert rc == 0
        return views

    def backproject(self, views, index=None):
        views = _c(views, self.dt)
        idx = None if index is None else np.ascontiguousarray(index, dtype=np.int32)
        n = self.nview if idx is None else len(idx)
        assert views.shape == (self.nx, self.nz, n)
        image = np.empty((self.nx, self.ny, self.nz), dtype=self.dt, order="F")
        fn = getattr(lib(), f"oracle_backproject_{self.sfx}")
        rc = fn(_ptr(image), _ptr(views), _ptr(self.mumap), _ptr(self.psfs), *self._args(),
                _ptr(idx), n, self.nthread)
        assert rc == 0
        return image

    def mlem(self, x0, y, bg, niter):
        out = np.empty((self.nx, self.ny, self.nz), dtype=self.dt, order="F")
        fn = getattr(lib(), f"oracle_mlem_{self.sfx}")
        rc = fn(_ptr(out), _ptr(_c(x0, self.dt)), _ptr(_c(y, self.dt)), _ptr(_c(bg, self.dt)),
                _ptr(self.mumap), _ptr(self.psfs), *self._args(), int(niter), self.nthread)
        assert rc == 0
        return out

    def osem(self, x0, y, bg, nblocks, niter):
        out = np.empty((self.nx, self.ny, self.nz), dtype=self.dt, order="F")
        fn = getattr(lib(), f"oracle_osem_{self.sfx}")
        rc = fn(_ptr(out), _ptr(_c(x0, self.dt)), _ptr(_c(y, self.dt)), _ptr(_c(bg, self.dt)),
                _ptr(self.mumap), _ptr(self.psfs), *self._args(), int(nblocks), int(niter), self.nthread)
        if rc != 0:
            raise ValueError("nview must be divisible by nblocks!")
        return out


def psf_gauss(ny=128, px=11, pz=None, fwhm_start=1.0, fwhm_end=4.0, fwhm=None, fwhm_x=None, fwhm_z=None,
              dtype=np.float32):
    """psf_gauss(; ny, px, pz, fwhm_start, fwhm_end, fwhm, fwhm_x, fwhm_z, T)
    restated in numpy (src/psf-gauss.jl:24-55): plane iy is the Float64
    outer product of two normalised 1-D Gaussians exp(-0.5 (r/sigma)^2),
    sigma = fwhm/sqrt(log 256), r = -(p-1)/2 .. (p-1)/2, rounded to T;
    fwhm == 0 gives the Kronecker impulse at r == 0.  fwhm defaults to
    range(fwhm_start, fwhm_end, ny) (numpy.linspace: same endpoints)."""
    pz = px if pz is None else pz
    if fwhm is None:
        fwhm = np.linspace(fwhm_start, fwhm_end, ny)
    fx = np.asarray(fwhm if fwhm_x is None else fwhm_x, dtype=np.float64)
    fz = np.asarray(fx if fwhm_z is None else fwhm_z, dtype=np.float64)

    def g(p, f):
        r = np.arange(-(p - 1) // 2, (p - 1) // 2 + 1, dtype=np.float64)
        if f == 0:
            if not (r == 0).any():
                raise ValueError("must have some r=0 if fwhm=0")
            return (r == 0).astype(np.float64)
        w = np.exp(-0.5 * (r / (f / np.sqrt(np.log(256.0)))) ** 2)
        return w / w.sum()

    out = np.empty((px, pz, ny), dtype=dtype, order="F")
    for iy in range(ny):
        out[:, :, iy] = np.outer(g(px, fx[iy]), g(pz, fz[iy])).astype(dtype)
    return out


def imrotate(img, theta, method="two", adj=False, dtype=np.float32):
    sfx, dt = _dt(dtype)
    img = _c(img, dt)
    n = img.shape[0]
    assert img.shape == (n, n)
    out = np.empty_like(img, order="F")
    getattr(lib(), f"oracle_imrotate_{sfx}")(_ptr(out), _ptr(img), n, float(theta),
                                             1 if method in ("one", 1) else 2, int(adj))
    return out


def fft_conv(img, ker, adj=False, dtype=np.float32):
    """img[nx,nz], ker[px,pz] (Julia order)."""
    sfx, dt = _dt(dtype)
    img = _c(img, dt)
    ker = _c(ker, dt)
    nx, nz = img.shape
    px, pz = ker.shape
    out = np.empty_like(img, order="F")
    getattr(lib(), f"oracle_fft_conv_{sfx}")(_ptr(out), _ptr(img), nx, nz, _ptr(ker), px, pz, int(adj))
    return out


def rot_f90(img, m, adj=False, dtype=np.float32):
    sfx, dt = _dt(dtype)
    img = _c(img, dt)
    out = np.empty_like(img, order="F")
    rc = getattr(lib(), f"oracle_rot_f90_{sfx}")(_ptr(out), _ptr(img), img.shape[0], int(m), int(adj))
    if rc != 0:
        raise ValueError("invalid m!")
    return out


def default_angles(nview, dtype=np.float32):
    sfx, dt = _dt(dtype)
    f = getattr(lib(), f"oracle_default_angle_{sfx}")
    return np.array([f(v, nview) for v in range(nview)], dtype=dt)


def padzero(img, pads):
    img = _c(img, np.float32)
    M, N = img.shape
    up, down, left, right = pads
    out = np.empty((M + up + down, N + left + right), np.float32, order="F")
    lib().oracle_padzero_f32(_ptr(out), _ptr(img), M, N, up, down, left, right)
    return out


def padrepl(img, pads):
    img = _c(img, np.float32)
    M, N = img.shape
    up, down, left, right = pads
    out = np.empty((M + up + down, N + left + right), np.float32, order="F")
    lib().oracle_padrepl_f32(_ptr(out), _ptr(img), M, N, up, down, left, right)
    return out


def pad2sizezero(img, padsize):
    img = _c(img, np.float32)
    M, N = img.shape
    P, Q = padsize
    out = np.empty((P, Q), np.float32, order="F")
    lib().oracle_pad2sizezero_f32(_ptr(out), _ptr(img), M, N, P, Q)
    return out


def fftshift2(img):
    img = _c(img, np.float32)
    M, N = img.shape
    out = np.empty_like(img, order="F")
    if lib().oracle_fftshift2_f32(_ptr(out), _ptr(img), M, N) != 0:
        raise ValueError("odd")
    return out


def rot_padsize(nx):
    return int(lib().oracle_rot_padsize(int(nx)))


def power2(x):
    return int(lib().oracle_power2(int(x)))
