"""Seeded synthetic SPECT studies (no public dataset exists for this path).

Each study follows the shapes and value distributions of the benchmark
workloads: ellipsoid emission phantoms (background 0.1 inside the
field of view, intensities U[0.5, 2]), ellipsoid attenuation maps in 1/mm
for a 4.8 mm voxel (0.0096/mm = 0.096/cm soft tissue, 0.015/mm = 0.15/cm,
0.004/mm lung-like), depth-dependent Gaussian PSFs from ``psf_gauss``
repeated over views (as in the reference's docs/lit/examples/1-overview.jl),
and Poisson data with a constant background of 5 % of the mean projection.
Everything is generated in float64 on the host from a fixed seed and stored
as float32 in the reference's column-major layout.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

BASE_SEED = 20261203


def ellipsoids(shape, k, rng, values, inside_fov_bg=None):
    """Sum of k random ellipsoids (centres in the central 60 %, semi-axes
    U[0.08, 0.3]*n, random rotation about z) on an (nx, ny, nz) grid."""
    nx, ny, nz = shape
    x = (np.arange(nx) - (nx - 1) / 2)[:, None, None]
    y = (np.arange(ny) - (ny - 1) / 2)[None, :, None]
    z = (np.arange(nz) - (nz - 1) / 2)[None, None, :]
    out = np.zeros(shape, np.float64)
    if inside_fov_bg is not None:
        r = np.sqrt(x ** 2 + y ** 2) + 0 * z
        out[r <= 0.45 * nx] = inside_fov_bg
    for i in range(k):
        cx, cy, cz = [rng.uniform(-0.3, 0.3) * n for n in shape]
        ax, ay, az = [rng.uniform(0.08, 0.3) * n for n in shape]
        phi = rng.uniform(0, np.pi)
        c, s = np.cos(phi), np.sin(phi)
        xr = c * (x - cx) + s * (y - cy)
        yr = -s * (x - cx) + c * (y - cy)
        mask = (xr / ax) ** 2 + (yr / ay) ** 2 + ((z - cz) / az) ** 2 <= 1
        out[mask] += values(i) if callable(values) else values
    return out


def body_mumap(shape, values, rng):
    """Attenuation map: a body ellipsoid of values[0], then nested/random
    ellipsoids of the other tissue values (in 1/mm)."""
    nx, ny, nz = shape
    x = (np.arange(nx) - (nx - 1) / 2)[:, None, None]
    y = (np.arange(ny) - (ny - 1) / 2)[None, :, None]
    z = (np.arange(nz) - (nz - 1) / 2)[None, None, :] + 0 * x + 0 * y
    mu = np.zeros(shape, np.float64)
    body = (x / (0.42 * nx)) ** 2 + (y / (0.34 * ny)) ** 2 <= 1
    mu[np.broadcast_to(body, shape)] = values[0]
    for v in values[1:]:
        cx, cy = rng.uniform(-0.12, 0.12) * nx, rng.uniform(-0.1, 0.1) * ny
        ax, ay, az = rng.uniform(0.08, 0.15) * nx, rng.uniform(0.08, 0.15) * ny, rng.uniform(0.2, 0.4) * nz
        m = ((x - cx) / ax) ** 2 + ((y - cy) / ay) ** 2 + (z / az) ** 2 <= 1
        mu[m & np.broadcast_to(body, shape)] = v
    return mu


@dataclass
class Study:
    name: str
    image: np.ndarray       # xtrue (nx, ny, nz)
    mumap: np.ndarray       # (nx, ny, nz), 1/mm
    psfs: np.ndarray        # (px, pz, ny, nview)
    dy: float               # mm
    nblocks: int = 1
    niter: int = 1
    ynoisy: np.ndarray | None = None
    background: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def nview(self):
        return self.psfs.shape[3]


def make_study(name, nx, nz, nview, p, fwhm_end, k, mu_values, nblocks, niter, seed, counts=None,
               project_fn=None, fwhm_start=1.0, psf_fn=None):
    """Build a study; ``project_fn(image, study) -> views`` supplies the
    noiseless data (the GPU projector or the oracle) for the Poisson draw.
    ``psf_fn`` is the psf_gauss generator (default: this package's host
    generator; a caller that must not load the CUDA library passes its own
    restatement, bit-identical by test)."""
    if psf_fn is None:
        from . import psf_gauss as psf_fn  # host generator, no GPU needed

    rng = np.random.default_rng(seed)
    shape = (nx, nx, nz)
    image = ellipsoids(shape, k, rng, lambda i: rng.uniform(0.5, 2.0), inside_fov_bg=0.1)
    mumap = body_mumap(shape, mu_values, rng)
    psf1 = psf_fn(ny=nx, px=p, fwhm_start=fwhm_start, fwhm_end=fwhm_end)
    psfs = np.asfortranarray(np.repeat(psf1[:, :, :, None], nview, axis=3))
    st = Study(name, np.asfortranarray(image, np.float32), np.asfortranarray(mumap, np.float32), psfs, 4.8,
               nblocks, niter, meta=dict(seed=seed, k=k, counts=counts))
    if project_fn is not None:
        ytrue = np.asarray(project_fn(st.image, st), dtype=np.float64)
        bg = 0.05 * ytrue.mean()
        if counts is None:
            y = rng.poisson(ytrue + bg).astype(np.float64)
            scale = 1.0
        else:
            scale = counts / (ytrue + bg).sum()
            y = rng.poisson(scale * (ytrue + bg)) / scale
        st.ynoisy = np.asfortranarray(y, np.float32)
        st.background = np.asfortranarray(np.full(ytrue.shape, bg), np.float32)
        st.meta["scale"] = scale
    return st


# Named studies (sizes, PSFs, attenuation, EM schedule) with their fixed seeds.
STUDIES = {
    "small_64x64x64": dict(nx=64, nz=64, nview=64, p=11, fwhm_end=3.0, k=4, mu_values=(0.0096,), nblocks=1,
                           niter=16),
    "larger_128x128x80": dict(nx=128, nz=80, nview=120, p=37, fwhm_end=6.0, k=8, mu_values=(0.0096, 0.015),
                              nblocks=8, niter=4, counts=1e6),
    "large_256x256x200": dict(nx=256, nz=200, nview=128, p=65, fwhm_end=10.0, k=12,
                              mu_values=(0.0096, 0.015, 0.004), nblocks=16, niter=4),
}
STUDY_SEED_OFFSET = {"small_64x64x64": 0, "larger_128x128x80": 1, "large_256x256x200": 4}


def named_study(name, project_fn=None, seed_offset=0, psf_fn=None):
    """The named study of STUDIES, generated from its fixed seed."""
    cfg = dict(STUDIES[name])
    return make_study(name, seed=BASE_SEED + STUDY_SEED_OFFSET[name] + seed_offset, project_fn=project_fn,
                      psf_fn=psf_fn, **cfg)


def divisors_in(n, lo=4, hi=16):
    return [d for d in range(lo, hi + 1) if n % d == 0]


def batch_mix(njobs, seed, big_fraction=0.0):
    """Uneven job mix of the batching/serving workloads: nx=ny in
    {64,96,128}, nz in [48,128], views in {60,90,120,128}, PSF in {11,21,37}
    (FWHM 1 -> p/6), OS-EM subsets from the divisors of nview in [4,16], and
    optionally a fraction of 256x256x128 jobs."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(njobs):
        if rng.uniform() < big_fraction:
            nx, nz = 256, 128
        else:
            nx = int(rng.choice([64, 96, 128]))
            nz = int(rng.integers(48, 129))
        nview = int(rng.choice([60, 90, 120, 128]))
        p = int(rng.choice([11, 21, 37]))
        nblocks = int(rng.choice(divisors_in(nview)))
        jobs.append(dict(nx=nx, nz=nz, nview=nview, p=p, fwhm_end=p / 6.0, k=int(rng.integers(4, 13)),
                         mu_values=(0.0096,), nblocks=nblocks, niter=4, seed=seed * 1000 + j))
    return jobs
