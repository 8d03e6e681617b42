"""Batched OS-EM (one CUDA-graph launch for many uneven reconstructions):
each job's result equals its own per-call osem! on the GPU and the oracle."""
import numpy as np
import pytest

from conftest import relerr

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _dev(torch, a):
    """Column-major host array -> device tensor exposing the same layout (x fastest)."""
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).cuda()
    return t.permute(*reversed(range(t.dim())))


def test_batch_matches_per_job(S, O):
    import importlib

    import torch

    W = importlib.import_module("spectrecon_b200.workloads")
    specs = [dict(nx=32, nz=24, nview=24, p=5, nblocks=4, niter=2),
             dict(nx=48, nz=20, nview=30, p=7, nblocks=5, niter=1),
             dict(nx=64, nz=40, nview=16, p=11, nblocks=8, niter=2)]
    plans, studies = [], []
    for j, sp in enumerate(specs):
        st = W.make_study(f"b{j}", nx=sp["nx"], nz=sp["nz"], nview=sp["nview"], p=sp["p"], fwhm_end=2.0, k=4,
                          mu_values=(0.0096,), nblocks=sp["nblocks"], niter=sp["niter"], seed=500 + j,
                          project_fn=lambda im, s: O.Geometry(s.mumap, s.psfs, s.dy).project(im))
        studies.append(st)
        plans.append(S.SPECTplan(st.mumap, st.psfs, st.dy))
    B = S.Batch(plans, [s["nblocks"] for s in specs], [s["niter"] for s in specs])
    outs = []
    for j, st in enumerate(studies):
        x0 = _dev(torch, np.ones(st.image.shape, np.float32))
        out = torch.zeros_like(x0)
        B.set_job(j, out, x0, _dev(torch, st.ynoisy), _dev(torch, st.background))
        outs.append(out)
    for _ in range(2):  # the graph is captured once and launched twice
        B.run()
    torch.cuda.synchronize()
    for j, st in enumerate(studies):
        got = outs[j].cpu().numpy()
        x0 = np.ones(st.image.shape, np.float32, order="F")
        ref_gpu = S.osem(x0, st.ynoisy, st.background, S.Ablock(plans[j], specs[j]["nblocks"]),
                         niter=specs[j]["niter"])
        ref_cpu = O.Geometry(st.mumap, st.psfs, st.dy).osem(x0, st.ynoisy, st.background, specs[j]["nblocks"],
                                                            specs[j]["niter"])
        assert relerr(got, ref_gpu) <= 1e-6
        assert relerr(got, ref_cpu) <= TOL
    B.close()
