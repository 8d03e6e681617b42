"""Generate the golden fixtures in tests/golden/ from the oracle.

The reference (Julia) cannot run on these machines, so the fixtures are
outputs of the oracle in float64 and float32 on fixed seeded inputs; the
oracle itself is pinned by the reference's known-answer and adjoint tests
(tests/test_oracle.py).  The fixtures freeze those outputs so that any later
change of the oracle or of the CUDA path is caught.  Re-run with
``python tests/golden/make_golden.py`` only when an intended change is made.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

CASES = {
    # name: (nx, nz, nview, px, pz, interp, mu_scale, seed)
    "small_two": (16, 12, 8, 5, 3, "two", 0.02, 101),
    "small_one": (16, 12, 8, 5, 3, "one", 0.02, 102),
    "odd_nz_two": (12, 7, 5, 7, 5, "two", 0.05, 103),
}


def inputs(nx, nz, nview, px, pz, mu_scale, seed):
    rng = np.random.default_rng(seed)
    mumap = np.asfortranarray(mu_scale * rng.random((nx, nx, nz)), np.float32)
    p = rng.random((px, pz, nx, nview))
    p = p + p[::-1, ::-1]
    psfs = np.asfortranarray(p / p.sum(axis=(0, 1), keepdims=True), np.float32)
    x = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    y = np.asfortranarray(rng.random((nx, nz, nview)), np.float32)
    return mumap, psfs, x, y


def main():
    for name, (nx, nz, nview, px, pz, interp, mus, seed) in CASES.items():
        mumap, psfs, x, y = inputs(nx, nz, nview, px, pz, mus, seed)
        out = dict(mumap=mumap, psfs=psfs, x=x, y=y, dy=np.float64(4.7952))
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            G = O.Geometry(mumap, psfs, 4.7952, interp=interp, dtype=dt, nthread=1)
            out[f"proj_{tag}"] = G.project(x)
            out[f"back_{tag}"] = G.backproject(y)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print("wrote", name)


if __name__ == "__main__":
    main()
