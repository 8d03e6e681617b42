"""B200-native SPECT projector behind SPECTrecon.jl's API (Python host mirror).

Mirrors the reference's public functions for the projector hot path with the
same names, argument meaning and errors; Julia's in-place ``f!`` becomes
``f_`` (the torch in-place convention):

=====================================  =======================================
reference (SPECTrecon.jl)              here
=====================================  =======================================
``SPECTplan(mumap, psfs, dy; ...)``    ``SPECTplan(mumap, psfs, dy, ...)``
``project!(views, image, plan; index)``  ``project_(views, image, plan, index=)``
``project(image, plan)``                ``project(image, plan)``
``project(image, mumap, psfs, dy)``     ``project(image, mumap, psfs, dy)``
``backproject!`` / ``backproject``      ``backproject_`` / ``backproject``
``mlem!`` / ``mlem``                    ``mlem_`` / ``mlem``
``osem!`` / ``osem``, ``Ablock``        ``osem_`` / ``osem``, ``Ablock``
``psf_gauss(; ...)``                    ``psf_gauss(...)``
=====================================  =======================================

Arrays use the reference's index order and memory layout: ``image[x,y,z]``
of shape ``(nx, ny, nz)``, ``views`` ``(nx, nz, nview)``, ``psfs``
``(px, pz, ny, nview)``, column-major (numpy ``order='F'``).  Host arrays are
numpy; device arrays are any object with ``__cuda_array_interface__`` (e.g. a
torch CUDA tensor) whose memory is column-major in that order.  View indices
are 0-based.  All compute runs in libspectgpu.so on the GPU; there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _native
from ._native import SpectError, check

__all__ = [
    "Batch", "Server", "SPECTplan", "project", "project_", "backproject", "backproject_", "mlem", "mlem_", "osem", "osem_",
    "Ablock", "psf_gauss", "psf_gauss_device", "nthreads", "SpectError",
]


def nthreads() -> int:
    """Analogue of ``Threads.nthreads()`` used by the ``nthread`` check."""
    return int(os.environ.get("SPECT_NTHREADS", os.cpu_count() or 1))


def _is_device(a) -> bool:
    return hasattr(a, "__cuda_array_interface__")


def _dev_ptr(a, shape, name):
    cai = a.__cuda_array_interface__
    if tuple(cai["shape"]) != tuple(shape):
        raise SpectError(8, f"DimensionMismatch: {name} has shape {tuple(cai['shape'])}, expected {tuple(shape)}")
    if cai["typestr"] not in ("<f4", "|f4"):
        raise TypeError(f"{name} must be float32 on the device")
    strides = cai.get("strides")
    want, s = [], 4
    for n in shape:
        want.append(s)
        s *= n
    if strides is not None and any(n > 1 and st != w for n, st, w in zip(shape, strides, want)):
        raise ValueError(f"{name} must be column-major (Julia layout) on the device")
    return cai["data"][0]


def _host_f32(a, shape, name):
    a = np.asarray(a)
    if a.shape != tuple(shape):
        raise SpectError(8, f"DimensionMismatch: {name} has shape {a.shape}, expected {tuple(shape)}")
    return np.asfortranarray(a, dtype=np.float32)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _index(index):
    if index is None:
        return None, None
    idx = np.ascontiguousarray(np.asarray(index, dtype=np.int32).ravel())
    return idx, _ptr(idx)


def _stream_ptr(stream):
    if stream is None:
        return None
    return getattr(stream, "cuda_stream", stream)


class SPECTplan:
    """System-model plan (src/spectplan.jl:58-137).

    ``SPECTplan(mumap, psfs, dy, T=np.float32, viewangle=None,
    interpmeth="two", nthread=nthreads(), mode="fast")`` validates the inputs
    exactly as the reference does and raises :class:`SpectError` with the
    reference's message ("nx != ny", "nx odd", "non-odd size psfs", "asym.
    psf", "bad interpmeth", "bad nthread", "bad mode").  ``mumap`` and
    ``psfs`` are host arrays; they are uploaded and the depth-dependent PSF
    spectra are precomputed on the GPU.  Unlike the reference plan (which
    aliases them), later edits of those arrays are not seen.
    """

    def __init__(self, mumap, psfs, dy, T=np.float32, viewangle=None, interpmeth="two", nthread=None, mode="fast"):
        if np.dtype(T) != np.float32:
            raise SpectError(13, f"T={np.dtype(T)}: the GPU path computes in Float32")
        mumap = np.asarray(mumap)
        psfs = np.asarray(psfs)
        if mumap.ndim != 3 or psfs.ndim != 4:
            raise SpectError(8, "DimensionMismatch: mumap must be 3-D and psfs 4-D")
        nx, ny, nz = mumap.shape
        px, pz, ny2, nview = psfs.shape
        if ny2 != ny and nx == ny:
            raise SpectError(8, "DimensionMismatch: image/psfs size")
        self.T = np.float32
        self.imgsize = (nx, ny, nz)
        self.px, self.pz, self.nview = px, pz, nview
        self.dy = np.float32(dy)
        self.interpmeth = {"one": 1, ":one": 1, 1: 1, "two": 2, ":two": 2, 2: 2}.get(interpmeth, -1)
        self.mode = {"fast": 0, ":fast": 0, "mem": 1, ":mem": 1}.get(mode, -1)
        self.nthread = nthreads() if nthread is None else int(nthread)
        mu = np.asfortranarray(mumap, dtype=np.float32)
        ps = np.asfortranarray(psfs, dtype=np.float32)
        ang = None
        if viewangle is not None:
            ang = np.ascontiguousarray(np.asarray(viewangle, dtype=np.float32).ravel())
            if ang.size != nview:
                raise SpectError(8, "DimensionMismatch: viewangle must have nview entries")
        self.viewangle = ang
        h = ctypes.c_void_p()
        check(_native.lib().spect_plan_create(
            ctypes.byref(h), nx, ny, nz, px, pz, nview, _ptr(mu), _ptr(ps), float(self.dy),
            None if ang is None else _ptr(ang), self.interpmeth, self.mode, self.nthread, nthreads()))
        self._h = h

    @classmethod
    def gauss(cls, mumap, dy, nview, px=11, pz=None, fwhm_start=1.0, fwhm_end=4.0, fwhm_z_start=None,
              fwhm_z_end=None, viewangle=None, interpmeth="two", nthread=None, mode="fast"):
        """SPECTplan(mumap, repeat(psf_gauss(; ny, px, pz, fwhm_start, fwhm_end),
        nview), dy) without building the PSF array: the Gaussian stack is
        generated on the GPU (spect_plan_create_gauss) and shared by all views."""
        pz = px if pz is None else pz
        fz0 = fwhm_start if fwhm_z_start is None else fwhm_z_start
        fz1 = fwhm_end if fwhm_z_end is None else fwhm_z_end
        mumap = np.asarray(mumap)
        if mumap.ndim != 3:
            raise SpectError(8, "DimensionMismatch: mumap must be 3-D")
        nx, ny, nz = mumap.shape
        self = cls.__new__(cls)
        self.T = np.float32
        self.imgsize = (nx, ny, nz)
        self.px, self.pz, self.nview = int(px), int(pz), int(nview)
        self.dy = np.float32(dy)
        self.interpmeth = {"one": 1, ":one": 1, 1: 1, "two": 2, ":two": 2, 2: 2}.get(interpmeth, -1)
        self.mode = {"fast": 0, ":fast": 0, "mem": 1, ":mem": 1}.get(mode, -1)
        self.nthread = nthreads() if nthread is None else int(nthread)
        mu = np.asfortranarray(mumap, dtype=np.float32)
        ang = None
        if viewangle is not None:
            ang = np.ascontiguousarray(np.asarray(viewangle, dtype=np.float32).ravel())
            if ang.size != nview:
                raise SpectError(8, "DimensionMismatch: viewangle must have nview entries")
        self.viewangle = ang
        h = ctypes.c_void_p()
        self._h = None
        check(_native.lib().spect_plan_create_gauss(
            ctypes.byref(h), nx, ny, nz, int(px), int(pz), int(nview), _ptr(mu), float(fwhm_start),
            float(fwhm_end), float(fz0), float(fz1), float(self.dy), None if ang is None else _ptr(ang),
            self.interpmeth, self.mode, self.nthread, nthreads()))
        self._h = h
        return self

    @property
    def handle(self):
        return self._h

    def info(self):
        out = (ctypes.c_int * 8)()
        b = ctypes.c_size_t()
        check(_native.lib().spect_plan_info(self._h, out, ctypes.byref(b)))
        keys = ("nx", "ny", "nz", "px", "pz", "nview", "interpmeth", "nset")
        d = dict(zip(keys, list(out)))
        d["device_bytes"] = b.value
        return d

    def conv_kernels(self):
        """Which convolution kernels the plan runs: {"forward": "direct" |
        "fft", "adjoint": ..., "direct_forward_ok": bool, "direct_adjoint_ok":
        bool}.  Direct kernels need rank-1 (separable) PSF planes; autotune()
        keeps whichever is faster for each direction."""
        out = (ctypes.c_int * 4)()
        check(_native.lib().spect_plan_conv_kernels(self._h, out))
        name = ("fft", "direct")
        return {"forward": name[out[2]], "adjoint": name[out[3]],
                "direct_forward_ok": bool(out[0]), "direct_adjoint_ok": bool(out[1])}

    @property
    def fused(self):
        """True when the plan runs the fused projector pair (rotation,
        attenuation, separable convolution and depth sum in one forward
        kernel; gather rotation adjoint with the EM update fused)."""
        out = ctypes.c_int(0)
        check(_native.lib().spect_plan_fused(self._h, ctypes.byref(out)))
        return out.value == 1

    @property
    def path(self):
        """Which kernels the plan runs: "fused" (the fused projector pair),
        "strip" (the same layouts and passes as one kernel per pass over plane
        tiles, for planes too large for the fused kernels' shared memory) or
        "split" (rotation, convolution and reduction kernels)."""
        out = ctypes.c_int(0)
        check(_native.lib().spect_plan_fused(self._h, ctypes.byref(out)))
        return ("split", "fused", "strip")[out.value]

    def conv_taps(self):
        """Mean PSF taps per depth plane that the z and x convolution passes
        run: the fused pair skips the outer taps below Float32 resolution of
        each plane's factors; other plans report (pz, px)."""
        out = (ctypes.c_double * 2)()
        check(_native.lib().spect_plan_fused_taps(self._h, out))
        return float(out[0]), float(out[1])

    def autotune(self, nindex=None):
        """Time candidate launch shapes for calls with nindex views (default
        nview) and keep the fastest; returns (forward_ms, adjoint_ms)."""
        ms = (ctypes.c_double * 2)()
        check(_native.lib().spect_plan_autotune(self._h, int(nindex or self.nview), ms))
        return ms[0], ms[1]

    def close(self):
        if getattr(self, "_h", None):
            _native.lib().spect_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __repr__(self):
        nx, ny, nz = self.imgsize
        return (f"SPECTplan{{Float32}} imgsize=({nx}, {ny}, {nz}) px={self.px} pz={self.pz} nview={self.nview} "
                f"interpmeth={'one' if self.interpmeth == 1 else 'two'} dy={self.dy}")


def _views_shape(plan, n):
    nx, _, nz = plan.imgsize
    return (nx, nz, n)


def project_(views, image, plan: SPECTplan, index=None, stream=None):
    """project!(views, image, plan; index) (src/project.jl:143-163).

    views[:,:,i] = P_{index[i]} image.  Host arrays: synchronous; device
    arrays: enqueued on ``stream``.  Returns ``views``.
    """
    idx, ip = _index(index)
    n = plan.nview if idx is None else idx.size
    L = _native.lib()
    if _is_device(views) or _is_device(image):
        vp = _dev_ptr(views, _views_shape(plan, n), "views")
        xp = _dev_ptr(image, plan.imgsize, "image")
        check(L.spect_project(plan.handle, vp, xp, ip, n, _stream_ptr(stream)))
        return views
    x = _host_f32(image, plan.imgsize, "image")
    if not (isinstance(views, np.ndarray) and views.dtype == np.float32 and views.flags.f_contiguous
            and views.shape == _views_shape(plan, n)):
        raise SpectError(8, f"DimensionMismatch: views must be a Float32 column-major array of shape "
                            f"{_views_shape(plan, n)}")
    check(L.spect_project_host(plan.handle, _ptr(views), _ptr(x), ip, n))
    return views


def backproject_(image, views, plan: SPECTplan, index=None, stream=None):
    """backproject!(image, views, plan; index) (src/backproject.jl:132-162)."""
    idx, ip = _index(index)
    n = plan.nview if idx is None else idx.size
    L = _native.lib()
    if _is_device(views) or _is_device(image):
        xp = _dev_ptr(image, plan.imgsize, "image")
        vp = _dev_ptr(views, _views_shape(plan, n), "views")
        check(L.spect_backproject(plan.handle, xp, vp, ip, n, _stream_ptr(stream)))
        return image
    v = _host_f32(views, _views_shape(plan, n), "views")
    if not (isinstance(image, np.ndarray) and image.dtype == np.float32 and image.flags.f_contiguous
            and image.shape == plan.imgsize):
        raise SpectError(8, f"DimensionMismatch: image must be a Float32 column-major array of shape {plan.imgsize}")
    check(L.spect_backproject_host(plan.handle, _ptr(image), _ptr(v), ip, n))
    return image


def project(image, plan_or_mumap, psfs=None, dy=None, interpmeth="two", mode="fast", index=None, **kw):
    """``project(image, plan; index)`` (src/project.jl:170-178) or
    ``project(image, mumap, psfs, dy; interpmeth, mode)`` (src/project.jl:194-208)."""
    if isinstance(plan_or_mumap, SPECTplan):
        plan = plan_or_mumap
    else:
        mumap = np.asarray(plan_or_mumap)
        if np.shape(mumap) != np.shape(image):
            raise SpectError(8, "DimensionMismatch: image/mumap size")
        if np.shape(image)[1] != np.shape(psfs)[2]:
            raise SpectError(8, "DimensionMismatch: image/psfs size")
        plan = SPECTplan(mumap, psfs, dy, interpmeth=interpmeth, mode=mode, **kw)
    n = plan.nview if index is None else len(np.ravel(index))
    views = np.empty(_views_shape(plan, n), dtype=np.float32, order="F")
    return project_(views, image, plan, index=index)


def backproject(views, plan_or_mumap, psfs=None, dy=None, interpmeth="two", mode="fast", index=None, **kw):
    """``backproject(views, plan; index)`` (src/backproject.jl:170-178) or
    ``backproject(views, mumap, psfs, dy; interpmeth, mode)`` (src/backproject.jl:187-203)."""
    if isinstance(plan_or_mumap, SPECTplan):
        plan = plan_or_mumap
    else:
        mumap = np.asarray(plan_or_mumap)
        views_a = np.asarray(views)
        if not (mumap.shape[0] == views_a.shape[0]):
            raise SpectError(8, "DimensionMismatch: nx")
        if mumap.shape[2] != views_a.shape[1]:
            raise SpectError(8, "DimensionMismatch: nz")
        plan = SPECTplan(mumap, psfs, dy, interpmeth=interpmeth, mode=mode, **kw)
    image = np.zeros(plan.imgsize, dtype=np.float32, order="F")
    return backproject_(image, views, plan, index=index)


class Ablock:
    """Ablock(plan, nblocks) (src/ml-os-em.jl:70-84): nblocks subsets of views
    nb:nblocks:nview (0-based here: b, b+nblocks, ...)."""

    def __init__(self, plan: SPECTplan, nblocks: int):
        if plan.nview % nblocks != 0:
            raise SpectError(10, "nview must be divisible by nblocks!")
        self.plan = plan
        self.nblocks = int(nblocks)
        self.index = [np.arange(b, plan.nview, nblocks, dtype=np.int32) for b in range(nblocks)]

    def __len__(self):
        return self.nblocks

    def __getitem__(self, b):
        return self.index[b]


def _em_common(out, x0, ynoisy, background, plan, nblocks, niter, stream):
    L = _native.lib()
    V = _views_shape(plan, plan.nview)
    if any(_is_device(a) for a in (out, x0, ynoisy, background)):
        po = _dev_ptr(out, plan.imgsize, "out")
        p0 = _dev_ptr(x0, plan.imgsize, "x0")
        py = _dev_ptr(ynoisy, V, "ynoisy")
        pb = _dev_ptr(background, V, "background")
        check(L.spect_osem(plan.handle, po, p0, py, pb, int(nblocks), int(niter), _stream_ptr(stream)))
        return out
    bg = np.asarray(background)
    if not np.all(bg > 0):
        raise SpectError(9, "need background > 0")
    if np.shape(out) != np.shape(x0):
        raise SpectError(8, "DimensionMismatch: size out and x0 not match")
    x = _host_f32(x0, plan.imgsize, "x0")
    y = _host_f32(ynoisy, V, "ynoisy")
    b = _host_f32(bg, V, "background")
    if not (isinstance(out, np.ndarray) and out.dtype == np.float32 and out.flags.f_contiguous):
        raise SpectError(8, "DimensionMismatch: out must be a Float32 column-major array")
    check(L.spect_osem_host(plan.handle, _ptr(out), _ptr(x), _ptr(y), _ptr(b), int(nblocks), int(niter)))
    return out


def mlem_(out, x0, ynoisy, background, A: SPECTplan, niter=20, chat=False, stream=None):
    """mlem!(out, x0, ynoisy, background, A; niter=20) (src/ml-os-em.jl:21-49)
    with A the plan's full system model; EM ratio and update fused on the GPU."""
    if np.shape(ynoisy) != np.shape(background):
        raise SpectError(8, "DimensionMismatch: size ynoisy and background")
    return _em_common(out, x0, ynoisy, background, A, 1, niter, stream)


def mlem(x0, ynoisy, background, A: SPECTplan, niter=20, chat=False):
    """mlem(x0, ynoisy, background, A; niter) (src/ml-os-em.jl:61)."""
    out = np.empty(A.imgsize, dtype=np.float32, order="F")
    return mlem_(out, x0, ynoisy, background, A, niter=niter, chat=chat)


def osem_(out, x0, ynoisy, background, Ab: Ablock, niter=16, chat=False, stream=None):
    """osem!(out, x0, ynoisy, background, Ab; niter=16) (src/ml-os-em.jl:97-131)."""
    return _em_common(out, x0, ynoisy, background, Ab.plan, Ab.nblocks, niter, stream)


def osem(x0, ynoisy, background, Ab: Ablock, niter=16, chat=False):
    """osem(x0, ynoisy, background, Ab; niter) (src/ml-os-em.jl:143)."""
    out = np.empty(Ab.plan.imgsize, dtype=np.float32, order="F")
    return osem_(out, x0, ynoisy, background, Ab, niter=niter, chat=chat)


class Batch:
    """Many OS-EM reconstructions of uneven sizes run as ONE CUDA-graph launch.

    ``Batch(plans, nblocks, niter)``; ``set_job(j, out, x0, ynoisy, background)``
    with device arrays (column-major like the reference); ``run(stream)``
    enqueues the whole batch (every job's osem!, src/ml-os-em.jl:97-131) as
    one graph launch.  No counterpart in the reference (one osem! at a time).
    """

    def __init__(self, plans, nblocks, niter):
        self.plans = list(plans)
        n = len(self.plans)
        nb = np.ascontiguousarray(np.broadcast_to(np.asarray(nblocks, np.int32), (n,)))
        ni = np.ascontiguousarray(np.broadcast_to(np.asarray(niter, np.int32), (n,)))
        self.nblocks, self.niter = nb, ni
        hs = (ctypes.c_void_p * n)(*[p.handle for p in self.plans])
        h = ctypes.c_void_p()
        check(_native.lib().spect_batch_create(ctypes.byref(h), n, hs, _ptr(nb), _ptr(ni)))
        self._h = h
        self._keep = {}

    def set_job(self, j, out, x0, ynoisy, background):
        p = self.plans[j]
        V = _views_shape(p, p.nview)
        ptrs = (_dev_ptr(out, p.imgsize, "out"), _dev_ptr(x0, p.imgsize, "x0"), _dev_ptr(ynoisy, V, "ynoisy"),
                _dev_ptr(background, V, "background"))
        self._keep[j] = (out, x0, ynoisy, background)
        check(_native.lib().spect_batch_set_job(self._h, int(j), *ptrs))

    def run(self, stream=None):
        check(_native.lib().spect_batch_run(self._h, _stream_ptr(stream)))

    def close(self):
        if getattr(self, "_h", None):
            _native.lib().spect_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching reconstruction server (no counterpart in the reference).

    ``Server(budget_bytes=0, max_active=16)``; ``submit(mumap, psfs, dy, ynoisy,
    background, nblocks, niter, x0=None, interpmeth="two")`` returns a ticket at
    once (host arrays in the reference's layout are copied); ``wait(ticket)``
    returns ``(image, latency_ms)``.  Admission is by device-memory budget and
    slots; admitted jobs keep their plan, spectra, attenuation and iterate on the
    GPU and run concurrently on their own streams.
    """

    def __init__(self, budget_bytes=0, max_active=16):
        h = ctypes.c_void_p()
        check(_native.lib().spect_server_create(ctypes.byref(h), int(budget_bytes), int(max_active)))
        self._h = h
        self._shapes = {}

    def submit(self, mumap, psfs, dy, ynoisy, background, nblocks, niter, x0=None, interpmeth="two"):
        mu = np.asfortranarray(mumap, np.float32)
        ps = np.asfortranarray(psfs, np.float32)
        nx, ny, nz = mu.shape
        px, pz, ny2, nview = ps.shape
        if nx != ny:
            raise SpectError(1, "nx != ny")
        if ny2 != ny:
            raise SpectError(8, "DimensionMismatch: image/psfs size")
        y = _host_f32(ynoisy, (nx, nz, nview), "ynoisy")
        b = _host_f32(background, (nx, nz, nview), "background")
        x = None if x0 is None else _host_f32(x0, (nx, ny, nz), "x0")
        d = _native.JobDesc(nx, nz, px, pz, nview, mu.ctypes.data, ps.ctypes.data, float(dy),
                            {"one": 1, "two": 2}.get(interpmeth, interpmeth), y.ctypes.data, b.ctypes.data,
                            None if x is None else x.ctypes.data, int(nblocks), int(niter))
        t = ctypes.c_longlong()
        check(_native.lib().spect_server_submit(self._h, ctypes.byref(d), ctypes.byref(t)))
        self._shapes[t.value] = (nx, ny, nz)
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        shape = self._shapes.pop(ticket)
        out = np.empty(shape, np.float32, order="F")
        lat = ctypes.c_double()
        check(_native.lib().spect_server_wait(self._h, ticket, _ptr(out), ctypes.byref(lat), int(timeout_ms)))
        return out, lat.value

    def stats(self):
        v = (ctypes.c_longlong * 8)()
        check(_native.lib().spect_server_stats(self._h, v))
        keys = ("submitted", "done", "failed", "active", "pending", "max_active_seen", "bytes_in_use", "budget")
        return dict(zip(keys, list(v)))

    def close(self):
        if getattr(self, "_h", None):
            _native.lib().spect_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def psf_gauss(ny=128, px=11, pz=None, fwhm_start=1, fwhm_end=4, fwhm=None, fwhm_x=None, fwhm_z=None,
              T=np.float32):
    """psf_gauss(; ny, px, pz, fwhm_start, fwhm_end, fwhm, fwhm_x, fwhm_z, T)
    (src/psf-gauss.jl:24-55): returns psf of shape (px, pz, ny), each plane
    the outer product of two normalised 1-D Gaussians (FWHM -> sigma =
    fwhm/sqrt(log 256)); fwhm == 0 gives a Kronecker impulse."""
    pz = px if pz is None else pz
    if fwhm is None:
        fwhm = np.linspace(fwhm_start, fwhm_end, ny)
    fx = np.ascontiguousarray(np.asarray(fwhm if fwhm_x is None else fwhm_x, dtype=np.float64))
    fz = np.ascontiguousarray(np.asarray(fx if fwhm_z is None else fwhm_z, dtype=np.float64))
    out = np.empty((px, pz, ny), dtype=np.float32, order="F")
    check(_native.lib().spect_psf_gauss(_ptr(out), int(ny), int(px), int(pz), _ptr(fx), _ptr(fz)))
    return out.astype(T, order="F")


def psf_gauss_device(out, ny=128, px=11, pz=None, fwhm_start=1.0, fwhm_end=4.0, fwhm_z_start=None,
                     fwhm_z_end=None, stream=None):
    """psf_gauss(; ny, px, pz, fwhm_start, fwhm_end) written on the GPU into
    ``out``, a float32 device array of shape (px, pz, ny) in column-major
    order (no host array, no allocation); returns ``out``."""
    pz = px if pz is None else pz
    fz0 = fwhm_start if fwhm_z_start is None else fwhm_z_start
    fz1 = fwhm_end if fwhm_z_end is None else fwhm_z_end
    p = _dev_ptr(out, (px, pz, ny), "psf")
    check(_native.lib().spect_psf_gauss_device(p, int(ny), int(px), int(pz), float(fwhm_start), float(fwhm_end),
                                               float(fz0), float(fz1), _stream_ptr(stream)))
    return out
