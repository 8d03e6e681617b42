"""Accuracy harness over MATLAB data files (accuracy/project.jl:1-60).

The reference's accuracy script reads four ``.mat`` files made with the MIRT
MATLAB toolbox -- ``mumap208.mat`` (variable ``mumap208``), ``psf_208.mat``
(``psf_208``), ``xtrue.mat`` (``xtrue``) and ``proj_jeff_newmumap.mat``
(``proj_jeff``) -- projects ``xtrue`` with every interpolation method and
memory mode, and prints the normalised RMS error of each projection set
against MIRT's (its notes: about 2e-7 for ``:one``, 4e-3 for ``:two``).  The
data files are not distributed with the reference; users supply them.

This module runs the same harness through the GPU projector.  ``.mat`` files
of MATLAB format versions 4 to 7 are read and written with ``scipy.io``;
version 7.3 files are HDF5 containers, which need ``h5py`` (absent here), and
are rejected with a message that says so.  The arrays keep MATLAB's index
order, which is the reference's (``image[x,y,z]``, ``views[x,z,view]``,
``psfs[x,z,y,view]``).  All projections compute in Float32: the reference
promotes its plan to the element type of the file's ``mumap`` (Float64 for
MATLAB doubles), the GPU path converts to Float32, which is far below the
interpolation errors the harness measures.
"""
from __future__ import annotations

import os

import numpy as np

__all__ = ["cal_nrmse", "read_mat", "write_mat", "load_project_data", "project_error", "PROJECT_FILES"]

#: file name and variable name of each input of the reference's harness (accuracy/project.jl:20-34)
PROJECT_FILES = {
    "mumap": ("mumap208.mat", "mumap208"),
    "psfs": ("psf_208.mat", "psf_208"),
    "xtrue": ("xtrue.mat", "xtrue"),
    "proj": ("proj_jeff_newmumap.mat", "proj_jeff"),
}

#: voxel size along the depth axis used by the harness (accuracy/project.jl:37)
PROJECT_DY = 4.7952


def cal_nrmse(x, xtrue) -> float:
    """Mean over the last axis of the per-slice relative 2-norm error
    ``||x[:,:,l] - xtrue[:,:,l]|| / ||xtrue[:,:,l]||`` (accuracy/project.jl:7-16).

    Both arrays must be 3-D with the same shape.  The sums run in Float64."""
    x = np.asarray(x)
    xtrue = np.asarray(xtrue)
    if x.ndim != 3 or x.shape != xtrue.shape:
        raise ValueError(f"cal_nrmse: shapes {x.shape} and {xtrue.shape} must be equal and 3-D")
    d = (x.astype(np.float64) - xtrue.astype(np.float64)).reshape(-1, x.shape[2], order="F")
    t = xtrue.astype(np.float64).reshape(-1, x.shape[2], order="F")
    return float(np.mean(np.linalg.norm(d, axis=0) / np.linalg.norm(t, axis=0)))


def _is_hdf5_mat(path) -> bool:
    """True for a MATLAB 7.3 file: its 116-byte text header names version 7.3."""
    with open(path, "rb") as f:
        return f.read(116).startswith(b"MATLAB 7.3")


def read_mat(path, name):
    """Variable ``name`` of the ``.mat`` file at ``path`` as a numpy array with
    MATLAB's index order (MAT.jl's ``read(matopen(path), name)``)."""
    import scipy.io

    if not os.path.isfile(path):
        raise FileNotFoundError(f"{path}: no such .mat file")
    if _is_hdf5_mat(path):
        raise ValueError(f"{path}: MATLAB 7.3 (HDF5) file; save it with -v7 or read it with h5py")
    d = scipy.io.loadmat(path, variable_names=[name])
    if name not in d:
        raise KeyError(f"{path} has no variable {name!r}")
    return np.asarray(d[name])


def write_mat(path, name, array) -> None:
    """Write ``array`` as variable ``name`` of a MATLAB 5/7 ``.mat`` file
    (MAT.jl's ``matwrite``); the index order is kept."""
    import scipy.io

    scipy.io.savemat(path, {name: np.asarray(array)}, do_compression=False)


def load_project_data(path):
    """The harness's four inputs from directory ``path``: a dict with
    ``mumap`` (nx,ny,nz), ``psfs`` (px,pz,ny,nview), ``xtrue`` (nx,ny,nz,
    converted to Float32 as the reference does) and ``proj`` (nx,nz,nview)."""
    out = {}
    for key, (fname, var) in PROJECT_FILES.items():
        out[key] = read_mat(os.path.join(path, fname), var)
    out["xtrue"] = np.asfortranarray(out["xtrue"], dtype=np.float32)
    nx, ny, nz = out["xtrue"].shape
    nview = out["psfs"].shape[3] if out["psfs"].ndim == 4 else -1
    if out["mumap"].shape != (nx, ny, nz) or out["psfs"].ndim != 4 or out["proj"].shape != (nx, nz, nview):
        raise ValueError(f"{path}: inconsistent shapes mumap {out['mumap'].shape}, psfs {out['psfs'].shape}, "
                         f"xtrue {out['xtrue'].shape}, proj {out['proj'].shape}")
    return out


def project_error(path="../data/", interpmeths=("one", "two"), modes=("fast", "mem"), dy=PROJECT_DY,
                  data=None, verbose=True):
    """accuracy/project.jl:18-55: for every interpolation method and mode,
    project ``xtrue`` through a plan of ``mumap`` and ``psfs`` on the GPU and
    return ``{(interpmeth, mode): nrmse}`` against the supplied projections.

    ``data`` (a dict as made by :func:`load_project_data`) replaces reading
    the files from ``path``."""
    from . import SPECTplan, project

    if data is None:
        data = load_project_data(path)
    out = {}
    for interpmeth in interpmeths:
        for mode in modes:
            if verbose:
                print(f"{interpmeth}, {mode}")
            plan = SPECTplan(data["mumap"], data["psfs"], dy, interpmeth=interpmeth, mode=mode)
            views = project(data["xtrue"], plan)
            nrmse = cal_nrmse(views, data["proj"])
            if verbose:
                print(f"nrmse = {nrmse}")
            out[(interpmeth, mode)] = nrmse
    return out
