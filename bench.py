"""Benchmark: OS-EM reconstructions per second on the single larger study.

Workload (one step = one full OS-EM reconstruction): image 128x128x80 Float32
with 8 random ellipsoids, attenuation map with two tissue values (0.15/cm and
0.096/cm, 4.8 mm voxels), 120 views over 360 degrees, 37x37 depth-dependent
Gaussian PSF (FWHM 1 -> 6 voxels), Poisson data at 1e6 total counts, OS-EM
with 8 subsets for 4 iterations (seeded synthetic data).

Our arm: ``value`` times spect_osem on device-resident inputs (CUDA events on
the launching stream, L2 flushed between steps); ``e2e`` times the host-array
C-ABI call spect_osem_host (pinned host buffers, H2D + D2H inside the timed
region).  ``--impl reference`` times the CPU oracle (the restatement of the
reference's threaded project!/backproject!/osem!; Julia is not installed):
every step one full OS-EM reconstruction of the same study on all host
threads, without loading the CUDA library.  ``cpu_baseline`` in our line is one
such reconstruction, and ``parity`` compares the GPU reconstruction timed here
with the Float32 and Float64 oracle reconstructions of the same inputs.

N > 1 (torchrun): the path does not exchange data between reconstructions,
so ranks run independent replicas (weak scaling, no collective on the data
path); ``value`` = all ranks' reconstructions / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "OS-EM recons/s batched+served vs plain (≤1e-4 rel err); p50/p99 latency; HBM GB/s"
WORKLOAD = ("single larger study: 128x128x80 f32, 8 ellipsoids, 2-value mumap, 120 views, 37x37 PSF "
            "FWHM 1-6, Poisson 1e6 counts, OS-EM 8 subsets x 4 iterations")
# the workload both arms run (identical in both JSON lines)
CONFIG = {"workload": WORKLOAD, "l2": "flushed between steps (256 MB write)", "parallelism": "replicas"}
KERNELS = ["k_rot_fwd", "k_conv_fwd", "k_reduce_views", "k_vspec", "k_conv_adj", "k_rot_adj", "k_reduce_image",
           "other"]


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def combine_ranks(total_ms, steps, backend="nccl"):
    """Max-over-ranks device time and the whole-job rate (replicas: every
    rank completes ``steps`` reconstructions)."""
    import torch
    import torch.distributed as dist

    ws = dist.get_world_size() if dist.is_initialized() else 1
    if ws > 1:
        t = torch.tensor([float(total_ms)], dtype=torch.float64,
                         device="cuda" if backend == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    return {"ms": total_ms, "value": ws * steps / (total_ms / 1e3)}


def fft_flops(nv, ny, Npx, Npz):
    """Algorithmic FLOPs of one projector pass over nv views: nv*ny*(5 N log2 N + 2 N),
    N = Npx*Npz (two real 2-D FFTs + a real-spectrum multiply per plane)."""
    N = Npx * Npz
    return nv * ny * (5.0 * N * np.log2(N) + 2.0 * N)


def direct_flops(nv, ny, nx, nz, px, pz):
    """Algorithmic FLOPs of one pass of the direct separable convolution over
    nv views: per plane a px-tap x pass and a pz-tap z pass over
    nx*nz samples, one FMA (2 FLOPs) per tap."""
    return nv * ny * 2.0 * nx * nz * (px + pz)


def read_traffic(name):
    """dram bytes per launch recorded in profiles/<name> (line 'traffic_bytes_per_launch: N')."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks(S, L):
    """Roofline denominators: the FP32 pipe measured here by the library's FFMA
    chain probe (spect_fp32_peak), and the HBM copy bandwidth of
    MEASURED_PEAKS.json when present (else the earlier pool measurement)."""
    fp = ctypes.c_double(0.0)
    S.check(L.spect_fp32_peak(ctypes.byref(fp)))
    hbm, src = 6650.0, "fallback (6.65 TB/s, earlier measurement on this pool)"
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        if m.get("hbm_gbs"):
            hbm, src = float(m["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, ValueError):
        pass
    return {"fp32_tflops": round(fp.value, 2), "fp32_source": "measured FFMA chains (spect_fp32_peak), this run",
            "hbm_gbs": hbm, "hbm_source": src}


PATH_NAMES = {"fused": "fused projector pair", "strip": "large-plane pass kernels", "split": "split kernels"}


def launch_work(plan, kind, nv):
    """(kernel name, bound, algorithmic FLOPs, algorithmic bytes, executed
    FLOPs or None) of one launch of kernel kind `kind` processing nv views,
    for the path the plan runs.  The algorithmic FLOPs of a convolution
    kernel are the fixed per-pass formula of the reference's algorithm (two
    real 2-D FFTs and a spectrum multiply per plane at its padded sizes,
    fft_flops), whatever this kernel does instead; the executed FLOPs are the
    FMAs it runs (1 FMA = 2 FLOP per kept tap of the z and x passes, plus the
    bilinear sample and attenuation).  The fused pair skips the outer taps
    below Float32 resolution of each plane's factors, so it counts the kept
    taps.  Bytes count each compulsory array once (attenuation planes,
    adjoint planes, images)."""
    nx, ny, nz = plan.imgsize
    px, pz = plan.px, plan.pz
    N, nxz = nx * ny * nz, nx * nz
    nzp = 16 * ((nz + 15) // 16)
    Npx = 1 << int(np.ceil(np.log2(nx + px - 1)))
    Npz = 1 << int(np.ceil(np.log2(nz + pz - 1)))
    F = fft_flops(nv, ny, Npx, Npz)
    path = plan.path
    if path == "strip":  # forward: two launches per pass (gather + z pass, x pass); adjoint: one
        tz, tx = plan.conv_taps()
        table = {
            "k_conv_fwd": ("k_zs_fz|k_zs_fx", "fp32", F / 2, 4.0 * (nv * ny * nx * nzp + N + 2 * nv * N) / 2,
                           nv * ny * nx * nz * (2.0 * (tx + tz) + 8) / 2),
            "k_conv_adj": ("k_zs_adj", "fp32", F, 4.0 * (2 * nv * ny * nx * nzp + nv * nxz),
                           nv * ny * nx * nz * (2.0 * (tx + tz) + 1)),
            "k_rot_adj": ("k_zrot_adj", "hbm", 8.0 * nv * N, 4.0 * (nv * ny * nx * nzp + 3 * N), None),
            "k_reduce_views": ("k_reduce_views", "hbm", 2.0 * nv * nxz, 4.0 * 4 * nv * nxz, None),
            "k_reduce_image": ("k_from_iz", "hbm", 0.0, 4.0 * 2 * N, None),
        }
    elif path == "fused":
        tz, tx = plan.conv_taps()
        table = {
            "k_conv_fwd": ("k_zfwd", "fp32", F, 4.0 * (nv * ny * nx * nzp + N), nv * ny * nx * nz * (2.0 * (tx + tz) + 8)),
            "k_conv_adj": ("k_zadj", "fp32", F, 4.0 * (2 * nv * ny * nx * nzp + nv * nxz),
                           nv * ny * nx * nz * (2.0 * (tx + tz) + 1)),
            "k_rot_adj": ("k_zrot_adj", "hbm", 8.0 * nv * N, 4.0 * (nv * ny * nx * nzp + 3 * N), None),
            "k_reduce_views": ("k_reduce_views", "hbm", 2.0 * nv * nxz, 4.0 * 4 * nv * nxz, None),
            "k_reduce_image": ("k_from_iz", "hbm", 0.0, 4.0 * 2 * N, None),
        }
    else:
        conv = plan.conv_kernels()
        ex = {"direct": direct_flops(nv, ny, nx, nz, px, pz), "fft": None}
        table = {
            "k_rot_fwd": ("k_rot_fwd", "hbm", 8.0 * nv * N, 4.0 * (N + nv * N), None),
            "k_conv_fwd": ("k_sconv_fwd" if conv["forward"] == "direct" else "k_conv_fwd2", "fp32",
                           F, 4.0 * (2 * nv * N), ex[conv["forward"]]),
            "k_conv_adj": ("k_sconv_adj" if conv["adjoint"] == "direct" else "k_conv_adj2", "fp32",
                           F, 4.0 * (2 * nv * N), ex[conv["adjoint"]]),
            "k_rot_adj": ("k_rot_adj", "hbm", 8.0 * nv * N, 4.0 * (nv * N + N), None),
            "k_reduce_views": ("k_reduce_views", "hbm", 2.0 * nv * nxz, 4.0 * 4 * nv * nxz, None),
            "k_reduce_image": ("k_reduce_image", "hbm", 0.0, 4.0 * 3 * N, None),
        }
    return table.get(kind)


def kernel_table(plan, kms, kn, steps, nv, pk, min_share=0.10):
    """Per-kernel time split and, for every kernel with at least `min_share`
    of the step, its roofline against its own bound: achieved = algorithmic
    work per launch / average CUDA-event launch time."""
    total = sum(kms.values()) or 1.0
    rows = []
    for k, ms in kms.items():
        if kn[k] == 0 or ms <= 0:
            continue
        w = launch_work(plan, k, nv)
        avg = ms / kn[k]
        row = {"kernel": w[0] if w else k, "ms_per_step": round(ms / steps, 3),
               "launches_per_step": int(kn[k] // steps), "share": round(ms / total, 3),
               "avg_launch_ms": round(avg, 4)}
        if w:
            name, bound, flops, nbytes, xflops = w
            tf = flops / (avg / 1e3) / 1e12
            gbs = nbytes / (avg / 1e3) / 1e9
            if bound == "fp32":
                row.update(bound="fp32", achieved=round(tf, 3), peak=pk["fp32_tflops"], unit="TFLOP/s",
                           frac=round(tf / pk["fp32_tflops"], 4))
                if xflops is not None:
                    xt = xflops / (avg / 1e3) / 1e12
                    row.update(executed_flops_per_launch=xflops, executed_tflops=round(xt, 3),
                               executed_frac=round(xt / pk["fp32_tflops"], 4))
            else:
                row.update(bound="hbm", achieved=round(gbs, 1), peak=pk["hbm_gbs"], unit="GB/s",
                           frac=round(gbs / pk["hbm_gbs"], 4))
            row.update(flops_per_launch=flops, algorithmic_bytes_per_launch=nbytes,
                       algorithmic_gbs=round(gbs, 1))
        rows.append(row)
    rows.sort(key=lambda r: -r["share"])
    return rows, [r for r in rows if r["share"] >= min_share and "bound" in r]


def build_study(S, plan_factory):
    from importlib import import_module

    W = import_module("spectrecon_b200.workloads")

    def proj(image, st):
        plan = plan_factory(st)
        v = S.project(image, plan)
        plan.close()
        return v

    return W.named_study("larger_128x128x80", project_fn=proj)


def run_ours(args):
    import torch

    import __graft_entry__ as GE

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    S = GE.load_package()
    L = S._native.lib()
    if args.study:  # one named study alone: its reconstructions/s, kernel split, rooflines, parity
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # 256 MB > 126 MB L2
        res = run_study(S, L, torch, args.study, args, peaks(S, L), flush)
        if rank == 0:
            print(json.dumps({"study": args.study, "unit": "recons/s", "higher_is_better": True, **res}), flush=True)
        return
    st = build_study(S, lambda s: S.SPECTplan(s.mumap, s.psfs, s.dy))
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    nx, ny, nz = plan.imgsize
    nview, nb, niter = st.nview, st.nblocks, st.niter
    tuned = plan.autotune(nview // nb)

    def dev(a):
        # column-major host array -> device tensor with the same memory order
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda()
        return t

    x0_h = np.ones((nx, ny, nz), np.float32, order="F")
    x0_d, y_d, b_d = dev(x0_h), dev(st.ynoisy), dev(st.background)
    out_d = torch.empty_like(x0_d)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # 256 MB > 126 MB L2

    def step():
        S.check(L.spect_osem(plan.handle, out_d.data_ptr(), x0_d.data_ptr(), y_d.data_ptr(), b_d.data_ptr(),
                             nb, niter, sp))

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    launches0 = L.spect_kernel_launches()
    S.check(L.spect_plan_profile(plan.handle, 1))
    times = []
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    if ws > 1:
        torch.distributed.barrier()
    launches = L.spect_kernel_launches() - launches0
    ms_k = (ctypes.c_double * 8)()
    n_k = (ctypes.c_longlong * 8)()
    S.check(L.spect_plan_kernel_times(plan.handle, ms_k, n_k))
    S.check(L.spect_plan_profile(plan.handle, 0))
    assert torch.isfinite(out_d).all().item()
    agg = combine_ranks(float(np.sum(times)), args.steps)
    total_ms, value = agg["ms"], agg["value"]

    # e2e: host arrays through the C ABI, pinned buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).pin_memory()
    x0_p, y_p, b_p = pin(x0_h), pin(st.ynoisy), pin(st.background)
    out_p = torch.empty_like(x0_p).pin_memory()

    def e2e_step():
        S.check(L.spect_osem_host(plan.handle, out_p.data_ptr(), x0_p.data_ptr(), y_p.data_ptr(), b_p.data_ptr(),
                                  nb, niter))

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    e2e_steps = max(1, args.steps)
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    etimes = []
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize()
        ev0.record()
        e2e_step()
        ev1.record()
        torch.cuda.synchronize()
        etimes.append(ev0.elapsed_time(ev1))
    agg = combine_ranks(float(np.sum(etimes)), e2e_steps)
    e2e_ms, e2e_value = agg["ms"], agg["value"]
    rel = float(np.abs(out_p.numpy().T - out_d.cpu().numpy().T).max() / np.abs(out_d.cpu().numpy()).max())

    # per-kernel split and rooflines (every kernel with >= 10 % of the step)
    kms = {k: ms_k[i] for i, k in enumerate(KERNELS)}
    kn = {k: n_k[i] for i, k in enumerate(KERNELS)}
    conv = plan.conv_kernels()
    nsub = nview // nb
    pk = peaks(S, L)
    split, roofs = kernel_table(plan, kms, kn, args.steps, nsub, pk)
    dom = dict(roofs[0]) if roofs else {}
    traffic = read_traffic(f"{dom.get('kernel')}_128x128x80.md") if dom else None
    roofline = dict(dom, traffic=traffic, traffic_source="ncu dram bytes per launch (profiles/)" if traffic else None,
                    peak_source=pk["fp32_source"] if dom.get("bound") == "fp32" else pk["hbm_source"])
    batched = served = None
    if not args.no_extras:
        batched = run_batched(S, torch)
        served = run_served(S, njobs=args.served_jobs, rate=args.served_rate)
    studies = None
    if not args.no_extras and ws == 1:
        studies = {n: run_study(S, L, torch, n, args, pk, flush) for n in ("small_64x64x64", "large_256x256x200")}
    cpu = parity = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        gpu_out = np.asfortranarray(out_d.cpu().numpy().T)
        cpu, parity = cpu_baseline(st, gpu_out)
    res = {
        "metric": METRIC, "value": round(value, 3), "unit": "recons/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantoms)",
        "config": dict(CONFIG),
        "path": PATH_NAMES[plan.path] + " (device-resident OS-EM), autotuned",
        "convolution": {"forward": conv["forward"], "adjoint": conv["adjoint"],
                        "taps_per_plane_z_x": [round(t, 2) for t in plan.conv_taps()], "psf_taps_z_x": [plan.pz, plan.px]},
        "parity": parity,
        "e2e": {"value": round(e2e_value, 3), "unit": "recons/s",
                "h2d_bytes_per_step": int(4 * (plan.imgsize[0] * ny * nz + 2 * nx * nz * nview)),
                "d2h_bytes_per_step": int(4 * nx * ny * nz), "ms_per_step": round(e2e_ms / e2e_steps, 3),
                "max_rel_diff_vs_device_path": rel},
        "gpu_launches": int(launches), "roofline": roofline, "kernels": roofs, "kernel_split": split,
        "peaks": pk, "clocks": clk.summary(), "cpu_baseline": cpu, "batched": batched, "served": served,
        "studies": studies,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)
    plan.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def plain_osem(S, plan, x0, y, bg, nblocks, niter):
    """The plain per-call GPU path: the reference's osem! loop (src/ml-os-em.jl:97-131)
    on host arrays, each project!/backproject! a synchronous C-ABI call with
    host<->device copies; ratio and update on the host."""
    Ab = S.Ablock(plan, nblocks)
    nx, _, nz = plan.imgsize
    ones = np.ones((nx, nz, plan.nview // nblocks), np.float32, order="F")
    asum = []
    for b in range(nblocks):
        a = S.backproject(ones, plan, index=Ab[b])
        a[a == 0] = np.inf
        asum.append(a)
    out = np.array(x0, dtype=np.float32, order="F", copy=True)
    for _ in range(niter):
        for b in range(nblocks):
            idx = Ab[b]
            ybar = S.project(out, plan, index=idx)
            yratio = y[:, :, idx] / (ybar + bg[:, :, idx])
            back = S.backproject(np.asfortranarray(yratio, np.float32), plan, index=idx)
            out *= back / asum[b]
    return out


def dev_f(torch, a):
    """Column-major host array -> device tensor with Julia layout (x fastest)."""
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).cuda()
    return t.permute(*reversed(range(t.dim())))


def run_batched(S, torch, njobs=32, timed_runs=2, plain_sample=6, seed=3):
    """Batching configuration: njobs reconstructions of uneven size (nx in
    {64,96,128}, nz in [48,128], views in {60,90,120,128}, PSF {11,21,37},
    4-16 subsets, 4 iterations) as one CUDA-graph launch, against the plain
    per-call path on a sample of the same jobs."""
    from importlib import import_module

    W = import_module("spectrecon_b200.workloads")
    jobs = W.batch_mix(njobs, seed)
    plans, studies = [], []
    for j in jobs:
        st = W.make_study("batch_job", nx=j["nx"], nz=j["nz"], nview=j["nview"], p=j["p"], fwhm_end=j["fwhm_end"],
                          k=j["k"], mu_values=j["mu_values"], nblocks=j["nblocks"], niter=j["niter"], seed=j["seed"],
                          project_fn=lambda im, s: S.project(im, S.SPECTplan(s.mumap, s.psfs, s.dy)))
        plans.append(S.SPECTplan(st.mumap, st.psfs, st.dy))
        studies.append(st)
    B = S.Batch(plans, [j["nblocks"] for j in jobs], [j["niter"] for j in jobs])
    outs, keep = [], []
    for k, st in enumerate(studies):
        x0 = dev_f(torch, np.ones(st.image.shape, np.float32))
        out = torch.zeros_like(x0)
        y, b = dev_f(torch, st.ynoisy), dev_f(torch, st.background)
        keep.append((x0, y, b))
        B.set_job(k, out, x0, y, b)
        outs.append(out)
    B.run()  # capture + first launch (warm-up)
    torch.cuda.synchronize()
    L = S._native.lib()
    l0 = L.spect_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(timed_runs):
        B.run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / timed_runs
    launches = (L.spect_kernel_launches() - l0) // timed_runs
    # the same jobs one after another through the device-resident spect_osem
    # (one call per job on one stream): what the graph adds over sequential
    # device-resident calls
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    seq_outs = [torch.zeros_like(o) for o in outs]

    def seq_all():
        for k, st in enumerate(studies):
            x0, y, b = keep[k]
            S.check(L.spect_osem(plans[k].handle, seq_outs[k].data_ptr(), x0.data_ptr(), y.data_ptr(), b.data_ptr(),
                                 jobs[k]["nblocks"], jobs[k]["niter"], sp))

    seq_all()
    torch.cuda.synchronize()
    e0.record()
    seq_all()
    e1.record()
    torch.cuda.synchronize()
    seq_ms = e0.elapsed_time(e1)
    seq_rel = max(float((a - b).abs().max() / b.abs().max()) for a, b in zip(outs, seq_outs))
    # plain per-call path on a sample of the jobs (wall clock: it is host driven)
    t_plain = []
    rel = 0.0
    for k in range(min(plain_sample, njobs)):
        st = studies[k]
        x0 = np.ones(st.image.shape, np.float32, order="F")
        t0 = time.perf_counter()
        ref = plain_osem(S, plans[k], x0, st.ynoisy, st.background, jobs[k]["nblocks"], jobs[k]["niter"])
        t_plain.append(time.perf_counter() - t0)
        got = outs[k].cpu().numpy()
        rel = max(rel, float(np.abs(got - ref).max() / np.abs(ref).max()))
    B.close()
    for p in plans:
        p.close()
    batched = njobs / (ms / 1e3)
    plain = 1.0 / float(np.mean(t_plain))
    return {"jobs": njobs, "recons_per_s": round(batched, 3), "ms_per_batch": round(ms, 2),
            "plain_percall_recons_per_s": round(plain, 3), "plain_sample_jobs": len(t_plain),
            "speedup_vs_plain": round(batched / plain, 2), "graph_kernels": int(launches),
            "max_rel_diff_vs_plain": rel,
            "sequential_device_recons_per_s": round(njobs / (seq_ms / 1e3), 3),
            "speedup_vs_sequential_device": round(batched / (njobs / (seq_ms / 1e3)), 2),
            "max_rel_diff_vs_sequential_device": seq_rel}


def run_served(S, njobs=500, rate=10.0, big_fraction=0.1, seed=4, pool_small=36, pool_big=3, plain_sample=10,
               saturated_jobs=150):
    """Serving configuration: a Poisson stream of reconstruction requests (the
    batching size mix plus big_fraction of 256x256x128 jobs, 4 OS-EM iterations
    each) submitted to the continuous-batching server at `rate` per second;
    p50/p99 submit-to-finish latency and throughput, a saturated run (all
    requests at once), and the plain per-call path on a sample of the mix."""
    from importlib import import_module

    W = import_module("spectrecon_b200.workloads")
    rng = np.random.default_rng(seed)
    mix = W.batch_mix(pool_small, seed)
    big = [dict(nx=256, nz=128, nview=int(rng.choice([60, 90, 120, 128])), p=int(rng.choice([11, 21, 37])),
                k=int(rng.integers(4, 13)), mu_values=(0.0096,), niter=4, seed=seed * 7919 + i) for i in range(pool_big)]
    for b in big:
        b["fwhm_end"] = b["p"] / 6.0
        b["nblocks"] = int(rng.choice(W.divisors_in(b["nview"])))
    pool = []
    for j in mix + big:
        st = W.make_study("served_job", nx=j["nx"], nz=j["nz"], nview=j["nview"], p=j["p"], fwhm_end=j["fwhm_end"],
                          k=j["k"], mu_values=j["mu_values"], nblocks=j["nblocks"], niter=j["niter"], seed=j["seed"])
        plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
        ytrue = S.project(st.image, plan).astype(np.float64)
        plan.close()
        bgv = 0.05 * ytrue.mean()
        st.background = np.asfortranarray(np.full(ytrue.shape, bgv), np.float32)
        st.meta["ytrue"] = ytrue
        pool.append(st)
    nsm = len(mix)
    picks = [int(rng.integers(nsm, len(pool))) if rng.uniform() < big_fraction else int(rng.integers(0, nsm))
             for _ in range(max(njobs, saturated_jobs))]
    ys = [np.asfortranarray(rng.poisson(pool[k].meta["ytrue"] + pool[k].background), np.float32) for k in picks]

    def stream(n, lam):
        srv = S.Server(max_active=24)
        arrivals = np.cumsum(rng.exponential(1.0 / lam, n)) if lam else np.zeros(n)
        tickets = []
        t0 = time.perf_counter()
        for i in range(n):
            while time.perf_counter() - t0 < arrivals[i]:
                time.sleep(min(0.002, max(0.0, arrivals[i] - (time.perf_counter() - t0))))
            st = pool[picks[i]]
            tickets.append(srv.submit(st.mumap, st.psfs, st.dy, ys[i], st.background, st.nblocks, st.niter))
        lat = [srv.wait(t)[1] for t in tickets]
        wall = time.perf_counter() - t0
        stats = srv.stats()
        srv.close()
        return lat, wall, stats

    lat, wall, stats = stream(njobs, rate)
    sat = [stream(saturated_jobs, None) for _ in range(3)]  # saturated, three times
    sat.sort(key=lambda r: r[1])
    slat, swall, sstats = sat[1]  # the median run
    # plain per-call path on a sample with the same share of big jobs
    nbig = max(1, int(round(plain_sample * big_fraction)))
    sample = [k for k in picks if k < nsm][: plain_sample - nbig] + [k for k in picks if k >= nsm][:nbig]
    # each served request builds its plan on the GPU, so the plain per-call
    # reconstruction is timed the same way: SPECTplan + osem! loop + release
    t_plain = 0.0
    for k in sample:
        st = pool[k]
        x0 = np.ones(st.image.shape, np.float32, order="F")
        y = np.asfortranarray(rng.poisson(st.meta["ytrue"] + st.background), np.float32)
        t0 = time.perf_counter()
        plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
        plain_osem(S, plan, x0, y, st.background, st.nblocks, st.niter)
        plan.close()
        t_plain += time.perf_counter() - t0
    plain = len(sample) / t_plain
    served = njobs / wall
    return {"requests": njobs, "arrival_rate_per_s": rate, "big_fraction": big_fraction,
            "recons_per_s": round(served, 3), "p50_ms": round(float(np.percentile(lat, 50)), 1),
            "p99_ms": round(float(np.percentile(lat, 99)), 1), "max_active": int(stats["max_active_seen"]),
            "failed": int(stats["failed"]),
            "saturated": {"requests": saturated_jobs, "recons_per_s": round(saturated_jobs / swall, 3),
                          "p50_ms": round(float(np.percentile(slat, 50)), 1),
                          "p99_ms": round(float(np.percentile(slat, 99)), 1),
                          "max_active": int(sstats["max_active_seen"]),
                          "runs": 3, "recons_per_s_min_med_max": [round(saturated_jobs / r[1], 3) for r in
                                                                  (sat[2], sat[1], sat[0])]},
            "plain_percall_recons_per_s": round(plain, 3), "plain_sample_jobs": len(sample),
            "plain_includes_plan_creation": True,
            "speedup_vs_plain": round(served / plain, 2),
            "saturated_speedup_vs_plain": round(saturated_jobs / swall / plain, 2)}


def run_study(S, L, torch, name, args, pk, flush):
    """One named study beside the benchmark line: device-resident
    reconstructions/s (CUDA events, L2 flushed), end to end through the host
    C-ABI call, the per-kernel split and rooflines, and the error of the GPU
    result against the Float32 and Float64 oracle -- the full reconstruction
    for the 64^3 ML-EM study (whose oracle run is also its CPU time), one
    OS-EM subset update (sensitivity of subset 0, then its update from a
    uniform start) for the 256x256x200 study, whose full oracle
    reconstruction would take tens of minutes."""
    from importlib import import_module

    from oracle import oracle as O

    W = import_module("spectrecon_b200.workloads")

    def proj(image, s):
        plan = S.SPECTplan(s.mumap, s.psfs, s.dy)
        v = S.project(image, plan)
        plan.close()
        return v

    st = W.named_study(name, project_fn=proj)
    plan = S.SPECTplan(st.mumap, st.psfs, st.dy)
    nx, ny, nz = plan.imgsize
    nb, niter = st.nblocks, st.niter
    nsub = st.nview // nb
    plan.autotune(nsub)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).cuda()
    x0_h = np.ones((nx, ny, nz), np.float32, order="F")
    x0_d, y_d, b_d = dev(x0_h), dev(st.ynoisy), dev(st.background)
    out_d = torch.empty_like(x0_d)
    stream = torch.cuda.current_stream()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def step():
        S.check(L.spect_osem(plan.handle, out_d.data_ptr(), x0_d.data_ptr(), y_d.data_ptr(), b_d.data_ptr(),
                             nb, niter, sp))

    for _ in range(max(3, args.warmup)):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    S.check(L.spect_plan_profile(plan.handle, 1))
    steps = max(3, min(args.steps, 10))
    times = []
    for _ in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms_k = (ctypes.c_double * 8)()
    n_k = (ctypes.c_longlong * 8)()
    S.check(L.spect_plan_kernel_times(plan.handle, ms_k, n_k))
    S.check(L.spect_plan_profile(plan.handle, 0))
    kms = {k: ms_k[i] for i, k in enumerate(KERNELS)}
    kn = {k: n_k[i] for i, k in enumerate(KERNELS)}
    split, roofs = kernel_table(plan, kms, kn, steps, nsub, pk)
    gpu_out = np.asfortranarray(out_d.cpu().numpy().T)
    # end to end: host arrays through the C ABI
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.float32).T)).pin_memory()
    x0_p, y_p, b_p = pin(x0_h), pin(st.ynoisy), pin(st.background)
    out_p = torch.empty_like(x0_p).pin_memory()
    e2e = []
    for r in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S.check(L.spect_osem_host(plan.handle, out_p.data_ptr(), x0_p.data_ptr(), y_p.data_ptr(), b_p.data_ptr(),
                                  nb, niter))
        if r:
            e2e.append(time.perf_counter() - t0)
    res = {"workload": f"{name}: {st.nview} views, {plan.px}x{plan.pz} PSF, "
                       f"{'ML-EM' if nb == 1 else f'OS-EM {nb} subsets'} x {niter} iterations",
           "path": PATH_NAMES[plan.path],
           "recons_per_s": round(1e3 * steps / float(np.sum(times)), 3), "ms_per_recon": round(float(np.mean(times)), 3),
           "e2e_recons_per_s": round(len(e2e) / float(np.sum(e2e)), 3),
           "h2d_bytes": int(4 * (nx * ny * nz + 2 * nx * nz * st.nview)), "d2h_bytes": int(4 * nx * ny * nz),
           "kernels": roofs, "kernel_split": split}
    if not args.no_cpu_baseline:
        if nb == 1:
            G32 = O.Geometry(st.mumap, st.psfs, st.dy)
            t0 = time.perf_counter()
            r32 = G32.mlem(x0_h, st.ynoisy, st.background, niter)
            t32 = time.perf_counter() - t0
            r64 = O.Geometry(st.mumap, st.psfs, st.dy, dtype=np.float64).mlem(x0_h, st.ynoisy, st.background, niter)
            res["cpu_oracle"] = {"recons_per_s": round(1.0 / t32, 5), "cores": os.cpu_count(),
                                 "sample": "one full ML-EM reconstruction, Float32, measured"}
            res["parity"] = {"what": "full reconstruction", "max_rel_vs_oracle_f32": float(np.abs(gpu_out - r32).max() / np.abs(r32).max()),
                             "max_rel_vs_oracle_f64": float(np.abs(gpu_out - r64).max() / np.abs(r64).max())}
        else:
            idx = np.arange(0, st.nview, nb, dtype=np.int32)
            asum_d, x_d = torch.empty_like(x0_d), dev(x0_h)
            ip = idx.ctypes.data_as(ctypes.c_void_p)
            S.check(L.spect_subset_sensitivity(plan.handle, asum_d.data_ptr(), ip, len(idx), sp))
            S.check(L.spect_em_subset_update(plan.handle, x_d.data_ptr(), y_d.data_ptr(), b_d.data_ptr(),
                                             asum_d.data_ptr(), ip, len(idx), sp))
            torch.cuda.synchronize()
            g1 = np.asfortranarray(x_d.cpu().numpy().T)
            par = {"what": f"one OS-EM subset update (views 0:{nb}:{st.nview}) from a uniform start"}
            for dt, key in ((np.float32, "max_rel_vs_oracle_f32"), (np.float64, "max_rel_vs_oracle_f64")):
                G = O.Geometry(st.mumap, st.psfs, st.dy, dtype=dt)
                ones = np.ones((nx, nz, len(idx)), dt, order="F")
                a = G.backproject(ones, index=idx)
                a = np.where(a == 0, np.inf, a)
                ybar = G.project(x0_h.astype(dt), index=idx)
                r = st.ynoisy[:, :, idx].astype(dt) / (ybar + st.background[:, :, idx].astype(dt))
                ref = x0_h.astype(dt) * (G.backproject(np.asfortranarray(r), index=idx) / a)
                par[key] = float(np.abs(g1 - ref).max() / np.abs(ref).max())
            res["parity"] = par
    plan.close()
    return res


def load_workloads():
    """spectrecon.jl_b200/workloads.py as a standalone module: the study
    generators without the package, so the CUDA library is not loaded."""
    import importlib.util

    name = "spect_workloads_standalone"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "spectrecon.jl_b200", "workloads.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def oracle_recon(st, dtype=np.float32, nthread=None):
    """One full OS-EM reconstruction of study ``st`` by the oracle (the
    restatement of the reference's threaded project!/backproject!/osem!,
    spawner-style chunking over views) on ``nthread`` host threads (default:
    all); returns (image, seconds)."""
    from oracle import oracle as O

    G = O.Geometry(st.mumap, st.psfs, st.dy, dtype=dtype, nthread=nthread or os.cpu_count())
    x0 = np.ones(st.mumap.shape, dtype, order="F")
    t0 = time.perf_counter()
    out = G.osem(x0, st.ynoisy, st.background, st.nblocks, st.niter)
    return out, time.perf_counter() - t0


def oracle_calibration():
    """The oracle on the reference's own timing case (time/project.jl:16-31:
    project! of a 64x64x40 image, 60 views, random symmetric 19x19 PSFs,
    :two, all threads), best of 3, beside the reference's published time for
    that call (289.8 ms, time/project.jl:60-61, on the reference authors'
    machine)."""
    from oracle import oracle as O

    rng = np.random.default_rng(0)
    nx, nz, nview, p = 64, 40, 60, 19
    mumap = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    psfs = rng.random((p, p, nx, nview))
    psfs = psfs + psfs[::-1, ::-1]
    psfs = psfs + psfs.transpose(1, 0, 2, 3)
    psfs = np.asfortranarray(psfs / psfs.sum(axis=(0, 1), keepdims=True), np.float32)
    G = O.Geometry(mumap, psfs, 4.7952)
    x = np.asfortranarray(rng.random((nx, nx, nz)), np.float32)
    best = 1e30
    for _ in range(3):
        t0 = time.perf_counter()
        G.project(x)
        best = min(best, time.perf_counter() - t0)
    return {"case": "project! 64x64x40, 60 views, 19x19 PSF, :two (time/project.jl)",
            "oracle_ms": round(1e3 * best, 1), "cores": os.cpu_count(), "reference_published_ms": 289.8}


def cpu_baseline(st, gpu_out=None):
    """The oracle on the host cores: one full Float32 OS-EM reconstruction of
    the benchmark study, measured (not extrapolated).  With ``gpu_out`` (the
    GPU reconstruction of the same inputs) also the parity of that
    reconstruction: max|gpu - oracle| / max|oracle| against the Float32 and
    the Float64 oracle."""
    out32, t32 = oracle_recon(st, np.float32)
    res = {"value": round(1.0 / t32, 6), "unit": "recons/s", "cores": os.cpu_count(), "kind": "port",
           "sample": f"one full OS-EM reconstruction of the same study ({st.nblocks} subsets x {st.niter} "
                     f"iterations, {st.nview} views), Float32, measured",
           "sample_seconds": round(t32, 2), "calibration": oracle_calibration()}
    parity = None
    if gpu_out is not None:
        out64, t64 = oracle_recon(st, np.float64)
        ref = np.abs(out64).max()
        parity = {"max_rel_vs_oracle_f32": float(np.abs(gpu_out - out32).max() / np.abs(out32).max()),
                  "max_rel_vs_oracle_f64": float(np.abs(gpu_out - out64).max() / ref),
                  "oracle_f32_vs_f64": float(np.abs(out32 - out64).max() / ref),
                  "tolerance": 1e-4,
                  "what": "the reconstruction timed above (full OS-EM), max|a-b|/max|b| over the image",
                  "oracle_f64_seconds": round(t64, 2)}
    return res, parity


def run_reference(args):
    """Reference arm: the oracle (the reference is Julia and cannot be installed
    here) runs the same study's full OS-EM on every host thread; each timed
    step is one complete reconstruction.  Warm-up steps each run one 15-view
    projection (the oracle keeps no state between calls)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as O

    W = load_workloads()

    def proj(image, s):
        return O.Geometry(s.mumap, s.psfs, s.dy).project(image)

    st = W.named_study("larger_128x128x80", project_fn=proj, psf_fn=O.psf_gauss)
    G = O.Geometry(st.mumap, st.psfs, st.dy)
    idx = np.arange(0, st.nview, st.nblocks, dtype=np.int32)
    x0 = np.ones(st.mumap.shape, np.float32, order="F")
    for _ in range(args.warmup):
        G.project(x0, index=idx)
    times = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        _, t = oracle_recon(st, np.float32)
        times.append(t)
    wall = time.perf_counter() - t0
    v = args.steps / float(np.sum(times))
    res = {"impl": "reference", "metric": METRIC, "value": round(v, 6), "unit": "recons/s", "n_gpus": ws,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * float(np.mean(times)), 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded phantoms)", "config": dict(CONFIG),
           "path": "CPU oracle: restatement of the reference's threaded project!/backproject!/osem! (no Julia)",
           "cpu_baseline": {"value": round(v, 6), "unit": "recons/s", "cores": os.cpu_count(), "kind": "port",
                            "sample": "every step one full OS-EM reconstruction of the study, measured",
                            "calibration": oracle_calibration()},
           "e2e": {"value": round(v, 6), "unit": "recons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "wall_s": round(wall, 1)}
    print(json.dumps(res), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batched/served measurements")
    ap.add_argument("--served-jobs", type=int, default=500)
    ap.add_argument("--served-rate", type=float, default=10.0)
    ap.add_argument("--study", choices=["small_64x64x64", "large_256x256x200"],
                    help="run only this study (the small 64^3 ML-EM or the large 256x256x200 OS-EM) and print its line")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
