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

    # roofline of the dominant kernel (FP32 pipe; the convolution, by FFT or
    # by the direct separable kernels, whichever the autotuner kept)
    kms = {k: ms_k[i] for i, k in enumerate(KERNELS)}
    kn = {k: n_k[i] for i, k in enumerate(KERNELS)}
    dom = max(("k_conv_fwd", "k_conv_adj"), key=lambda k: kms[k])
    conv = plan.conv_kernels()
    direct = conv["forward" if dom == "k_conv_fwd" else "adjoint"] == "direct"
    Npx = 1 << int(np.ceil(np.log2(nx + plan.px - 1)))
    Npz = 1 << int(np.ceil(np.log2(nz + plan.pz - 1)))
    nsub = nview // nb
    if direct:
        flops_launch = direct_flops(nsub, ny, nx, nz, plan.px, plan.pz)
        kname = dom.replace("k_conv", "k_sconv")
    else:
        flops_launch = fft_flops(nsub, ny, Npx, Npz)
        kname = dom
    avg_ms = kms[dom] / max(kn[dom], 1)
    achieved = flops_launch / (avg_ms / 1e3) / 1e12
    peak = measure_fp32_peak(torch)
    traffic = read_traffic(f"{kname}_c2.md")
    roofline = {"bound": "fp32", "achieved": round(achieved, 3), "peak": round(peak, 2), "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "kernel": kname,
                "convolution": conv["forward" if dom == "k_conv_fwd" else "adjoint"],
                "peak_source": "measured cuBLAS SGEMM (TF32 off) in this run",
                "flops_per_launch": flops_launch, "avg_launch_ms": round(avg_ms, 4),
                # DRAM bytes of one launch (ncu capture in profiles/) over its live duration
                "hbm_gbs": round(traffic / (avg_ms / 1e3) / 1e9, 1) if traffic and avg_ms > 0 else None,
                "kernel_ms_per_step": {k: round(v / args.steps, 3) for k, v in kms.items()},
                "kernel_launches_per_step": {k: int(v // args.steps) for k, v in kn.items()}}
    batched = served = None
    if not args.no_extras:
        batched = run_batched(S, torch)
        served = run_served(S, njobs=args.served_jobs, rate=args.served_rate)
    cpu = parity = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        gpu_out = np.asfortranarray(out_d.cpu().numpy().T)
        cpu, parity = cpu_baseline(st, gpu_out)
    res = {
        "metric": METRIC, "value": round(value, 3), "unit": "recons/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantoms)",
        "config": dict(CONFIG), "path": "fused OS-EM (device-resident), autotuned launch shapes",
        "convolution": {"forward": conv["forward"], "adjoint": conv["adjoint"]}, "parity": parity,
        "e2e": {"value": round(e2e_value, 3), "unit": "recons/s",
                "h2d_bytes_per_step": int(4 * (plan.imgsize[0] * ny * nz + 2 * nx * nz * nview)),
                "d2h_bytes_per_step": int(4 * nx * ny * nz), "ms_per_step": round(e2e_ms / e2e_steps, 3),
                "max_rel_diff_vs_device_path": rel},
        "gpu_launches": int(launches), "roofline": roofline, "clocks": clk.summary(),
        "cpu_baseline": cpu, "batched": batched, "served": served,
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
            "max_rel_diff_vs_plain": rel}


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
    slat, swall, sstats = stream(saturated_jobs, None)
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
                          "max_active": int(sstats["max_active_seen"])},
            "plain_percall_recons_per_s": round(plain, 3), "plain_sample_jobs": len(sample),
            "plain_includes_plan_creation": True,
            "speedup_vs_plain": round(served / plain, 2),
            "saturated_speedup_vs_plain": round(saturated_jobs / swall / plain, 2)}


def measure_fp32_peak(torch):
    """FP32 (non-tensor) peak: cuBLAS SGEMM 8192^3 with TF32 disabled, best of 5."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda")
    b = torch.randn(n, n, device="cuda")
    c = a @ b
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) / 1e3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b, c
    return best


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
           "sample_seconds": round(t32, 2)}
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
                            "sample": "every step one full OS-EM reconstruction of the study, measured"},
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
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
