"""Host-side tests that need no GPU: the C ABI library, argument validation
(the reference's error messages), psf_gauss, the workload generator and the
multi-process (gloo) replica aggregation used by bench.py."""
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "spect_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(spect_\w+)\s*\(", src)))


def test_library_exports_every_header_symbol(S):
    L = S._native.lib()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(S._native.symbols())


def test_julia_shim_binds_declared_symbols():
    """Every ccall of the Julia shim names a function that include/spect_gpu.h
    declares (the shim cannot run here: no Julia)."""
    src = open(os.path.join(ROOT, "spectrecon.jl_b200", "julia", "SPECTreconB200.jl")).read()
    called = set(re.findall(r"ccall\(\(:(spect_\w+),", src))
    assert {"spect_plan_create", "spect_project_host", "spect_backproject_host", "spect_osem_host"} <= called
    assert called <= set(header_functions()), called - set(header_functions())


def test_build_targets_sm100a():
    import __graft_entry__ as GE
    assert "arch=compute_100a,code=sm_100a" in GE.NVCC_FLAGS


def _psfs(px=3, pz=3, ny=8, nview=2):
    p = np.ones((px, pz, ny, nview), np.float32)
    return p / p[:, :, 0, 0].sum()


@pytest.mark.parametrize("mumap,psfs,kw,msg", [
    (np.zeros((8, 6, 4)), _psfs(ny=6), {}, "nx != ny"),
    (np.zeros((7, 7, 4)), _psfs(ny=7), {}, "nx odd"),
    (np.zeros((8, 8, 4)), np.ones((4, 3, 8, 2)), {}, "non-odd size psfs"),
    (np.zeros((8, 8, 4)), np.arange(9 * 8 * 2, dtype=np.float32).reshape((3, 3, 8, 2)), {}, "asym. psf"),
    (np.zeros((8, 8, 4)), _psfs(), {"interpmeth": "three"}, "bad interpmeth"),
    (np.zeros((8, 8, 4)), _psfs(), {"nthread": 10 ** 6}, "bad nthread"),
    (np.zeros((8, 8, 4)), _psfs(), {"mode": "slow"}, "bad mode"),
])
def test_plan_validation_messages(S, mumap, psfs, kw, msg):
    """SPECTplan throws the reference's strings (src/spectplan.jl:76-93)."""
    with pytest.raises(S.SpectError) as e:
        S.SPECTplan(mumap, psfs, 4.0, **kw)
    assert str(e.value) == msg


def test_psf_gauss_known_answers(S):  # test/psf-gauss.jl:7-31
    psf = S.psf_gauss()
    assert psf.dtype == np.float32 and psf.shape == (11, 11, 128)
    ny, px, pz = 4, 5, 3
    psf = S.psf_gauss(ny=ny, px=px, pz=pz, fwhm=np.zeros(ny))
    tmp = np.zeros((px, pz))
    tmp[(px - 1) // 2, (pz - 1) // 2] = 1
    assert np.array_equal(psf, np.repeat(tmp[:, :, None], ny, axis=2))
    psf = S.psf_gauss(ny=ny, px=px, pz=pz, fwhm_x=np.full(ny, np.inf), fwhm_z=np.zeros(ny))
    tmp = np.zeros((px, pz))
    tmp[:, (pz - 1) // 2] = 1 / px
    assert np.allclose(psf, np.repeat(tmp[:, :, None], ny, axis=2))


def test_psf_gauss_matches_definition(S):
    ny, px = 6, 9
    psf = S.psf_gauss(ny=ny, px=px, fwhm_start=1, fwhm_end=4)
    r = np.arange(px) - (px - 1) // 2
    for iy, f in enumerate(np.linspace(1, 4, ny)):
        s = f / np.sqrt(np.log(256))
        w = np.exp(-0.5 * (r / s) ** 2)
        w /= w.sum()
        assert np.allclose(psf[:, :, iy], np.outer(w, w), rtol=1e-6, atol=1e-8)
        assert abs(psf[:, :, iy].sum() - 1) < 1e-5
        assert np.array_equal(psf[:, :, iy], psf[::-1, ::-1, iy])  # point-symmetric, accepted by SPECTplan


def test_ablock_subsets(S):
    class P:
        nview = 12
    ab = S.Ablock(P(), 4)
    assert [list(ab[b]) for b in range(4)] == [[0, 4, 8], [1, 5, 9], [2, 6, 10], [3, 7, 11]]
    with pytest.raises(S.SpectError) as e:
        S.Ablock(P(), 5)
    assert str(e.value) == "nview must be divisible by nblocks!"


def test_em_background_check(S):
    class P:
        imgsize = (4, 4, 2)
        nview = 2
    bg = np.zeros((4, 2, 2), np.float32)
    with pytest.raises(S.SpectError) as e:
        S._em_common(np.zeros((4, 4, 2), np.float32), np.ones((4, 4, 2), np.float32), bg, bg, P(), 1, 1, None)
    assert str(e.value) == "need background > 0"


def test_workloads_seeded(S):
    import importlib
    W = importlib.import_module("spectrecon_b200.workloads")
    a = W.named_study("small_64x64x64")
    b = W.named_study("small_64x64x64")
    assert np.array_equal(a.image, b.image) and np.array_equal(a.mumap, b.mumap)
    assert a.image.shape == (64, 64, 64) and a.psfs.shape == (11, 11, 64, 64)
    assert a.image.min() >= 0 and 0.5 < a.image.max() <= 2.1 + 12 * 2
    assert set(np.unique(a.mumap)) <= {0.0, np.float32(0.0096)}
    for j in W.batch_mix(32, 5):
        assert j["nview"] % j["nblocks"] == 0 and 4 <= j["nblocks"] <= 16


def test_replica_aggregation_gloo():
    """bench.py's N>1 path (replicas, max-over-ranks timing) on 2 gloo ranks."""
    env = dict(os.environ, ROOT=ROOT, MASTER_ADDR="127.0.0.1", MASTER_PORT="29517")
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                          "--master-addr", "127.0.0.1", "--master-port", "29517",
                          os.path.join(ROOT, "tests", "_gloo_replicas.py")],
                         env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr[-2000:]
    assert out.stdout.count("ok") == 2


_C_CALLER = r"""
#include <math.h>
#include <stdio.h>
#include <string.h>
#include "spect_gpu.h"

int main(void) {
  enum { NY = 4, PX = 5, PZ = 3 };
  float psf[NY * PZ * PX];
  double fx[NY] = {0.0, 1.0, 2.0, 3.0}, fz[NY] = {0.0, 1.5, 1.5, 2.5};
  float mumap[8 * 6 * 4] = {0}, psfs[3 * 3 * 6 * 2];
  spect_plan_t plan = NULL;
  int y, i, rc;
  if (spect_psf_gauss(psf, NY, PX, PZ, fx, fz) != SPECT_OK) return 1;
  for (y = 0; y < NY; ++y) {
    double s = 0.0;
    for (i = 0; i < PX * PZ; ++i) s += psf[y * PX * PZ + i];
    if (fabs(s - 1.0) > 1e-6) return 2;
  }
  /* fwhm 0 on both axes: the impulse at the centre (test/psf-gauss.jl) */
  if (psf[(PZ / 2) * PX + PX / 2] != 1.0f) return 3;
  for (i = 0; i < 3 * 3 * 6 * 2; ++i) psfs[i] = 1.0f / 9.0f;
  /* nx = 8 != ny = 6: the reference's throw string, no device needed */
  rc = spect_plan_create(&plan, 8, 6, 4, 3, 3, 2, mumap, psfs, 4.8f, NULL, SPECT_INTERP_TWO,
                         SPECT_MODE_FAST, 1, 1);
  if (rc != SPECT_ERR_NX_NE_NY || strstr(spect_last_error(), "nx != ny") == NULL) return 4;
  if (spect_psf_gauss(NULL, NY, PX, PZ, fx, fz) == SPECT_OK) return 5;
  printf("ok\n");
  return 0;
}
"""


def test_c_caller_compiles_and_runs(S, tmp_path):
    """A C99 caller of include/spect_gpu.h (the boundary that Julia's ccall
    and C hosts bind) compiles without warnings, links libspectgpu.so and
    gets the host generator's results and the reference's error text
    without touching a device."""
    import shutil

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lib = os.path.join(ROOT, "spectrecon.jl_b200", "libspectgpu.so")
    S._native.lib()  # builds the library when missing
    src = tmp_path / "caller.c"
    src.write_text(_C_CALLER)
    exe = tmp_path / "caller"
    cmd = [cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
           str(src), "-o", str(exe), lib, f"-Wl,-rpath,{os.path.dirname(lib)}", "-lm"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.strip() == "ok"
