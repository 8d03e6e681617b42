"""Accuracy harness over .mat files (accuracy/project.jl of the reference).

The reference's data files come from MATLAB and are not distributed, so the
tests write seeded stand-ins with the same file and variable names: the CPU
tests check the file handling and the error measure, the GPU test runs the
whole harness with the oracle's projections in place of MIRT's.
"""
import importlib
import os

import numpy as np
import pytest

from conftest import sym_psfs


@pytest.fixture(scope="module")
def A(S):
    return importlib.import_module("spectrecon_b200.accuracy")


def _dataset(tmp_path, A, mumap, psfs, xtrue, proj):
    for key, arr in (("mumap", mumap), ("psfs", psfs), ("xtrue", xtrue), ("proj", proj)):
        fname, var = A.PROJECT_FILES[key]
        A.write_mat(os.path.join(tmp_path, fname), var, arr)
    return str(tmp_path)


def test_cal_nrmse_definition(A):
    """Per-slice relative 2-norm error averaged over the last axis (accuracy/project.jl:7-16)."""
    rng = np.random.default_rng(7)
    t = rng.random((6, 5, 4))
    x = t + 0.01 * rng.standard_normal(t.shape)
    want = np.mean([np.linalg.norm(x[:, :, l] - t[:, :, l]) / np.linalg.norm(t[:, :, l]) for l in range(4)])
    assert A.cal_nrmse(x, t) == pytest.approx(want, rel=1e-12)
    assert A.cal_nrmse(t, t) == 0.0
    with pytest.raises(ValueError):
        A.cal_nrmse(x[:, :, :3], t)


def test_mat_round_trip_keeps_index_order(A, tmp_path):
    rng = np.random.default_rng(8)
    a = np.asfortranarray(rng.random((6, 4, 3)), np.float32)
    p = os.path.join(tmp_path, "a.mat")
    A.write_mat(p, "vol", a)
    b = A.read_mat(p, "vol")
    assert b.shape == (6, 4, 3) and b.dtype == np.float32
    assert np.array_equal(a, b)
    with pytest.raises(KeyError):
        A.read_mat(p, "other")
    with pytest.raises(FileNotFoundError):
        A.read_mat(os.path.join(tmp_path, "missing.mat"), "vol")


def test_hdf5_mat_rejected(A, tmp_path):
    p = os.path.join(tmp_path, "v73.mat")
    with open(p, "wb") as f:
        f.write(b"MATLAB 7.3 MAT-file, Platform: GLNXA64".ljust(128, b" ") + b"\x89HDF\r\n\x1a\n")
    with pytest.raises(ValueError, match="7.3"):
        A.read_mat(p, "xtrue")


def test_load_project_data_shapes(A, tmp_path):
    rng = np.random.default_rng(9)
    nx, nz, nview = 8, 4, 6
    mumap = rng.random((nx, nx, nz))
    psfs = sym_psfs(rng, 3, 3, nx, nview).astype(np.float64)
    xtrue = rng.random((nx, nx, nz))
    proj = rng.random((nx, nz, nview))
    d = A.load_project_data(_dataset(tmp_path, A, mumap, psfs, xtrue, proj))
    assert d["xtrue"].dtype == np.float32 and d["xtrue"].flags.f_contiguous
    assert d["psfs"].shape == (3, 3, nx, nview) and d["proj"].shape == (nx, nz, nview)
    A.write_mat(os.path.join(tmp_path, "proj_jeff_newmumap.mat"), "proj_jeff", proj[:, :, :5])
    with pytest.raises(ValueError, match="inconsistent shapes"):
        A.load_project_data(str(tmp_path))


@pytest.mark.gpu
def test_project_error_harness(A, O, tmp_path):
    """The whole harness on a seeded 32x32x16 study with 12 views and 5x5
    PSFs, MATLAB doubles on disk as in the reference's data.  With the Float64
    oracle's projections standing in for MIRT's, every interpolation method
    and mode agrees with the oracle of the same method to <= 1e-5 nrmse, and
    :one against :two shows the interpolation gap the harness exists to
    measure (well above Float32 rounding)."""
    rng = np.random.default_rng(20261204)
    nx, nz, nview = 32, 16, 12
    mumap = 0.02 * rng.random((nx, nx, nz))
    psfs = sym_psfs(rng, 5, 5, nx, nview).astype(np.float64)
    xtrue = rng.random((nx, nx, nz))
    dy = A.PROJECT_DY
    ref = {m: O.Geometry(mumap, psfs, dy, interp=m, dtype=np.float64).project(xtrue) for m in ("one", "two")}
    path = _dataset(tmp_path, A, mumap, psfs, xtrue, ref["one"])
    err = A.project_error(path, verbose=False)
    assert set(err) == {(m, md) for m in ("one", "two") for md in ("fast", "mem")}
    assert err[("one", "fast")] <= 1e-5 and err[("one", "mem")] <= 1e-5
    assert 1e-4 < err[("two", "fast")] < 0.1
    data = A.load_project_data(path)
    data["proj"] = ref["two"]
    err2 = A.project_error(interpmeths=("two",), data=data, verbose=False)
    assert err2[("two", "fast")] <= 1e-5 and err2[("two", "mem")] <= 1e-5
