#!/usr/bin/env python3
"""Benchmark: patches/s per K-SVD iteration (OMP + dictionary update).

Workload (default): one 2048 x 2048 synthetic grayscale image (seeded
gratings + flat rectangles, Gaussian noise sigma 25), 12 x 12 patches at
stride 3 (679^2 = 461,041 patches of 144 values), 256 atoms, OMP limited to
5 atoms, 10 K-SVD iterations for the end-to-end call.

A "step" is one K-SVD iteration over all patches (kSvd's loop body,
cuda_svd_denoiser.cu:374-397).  value = patches x steps / device time of the
steps (max over ranks), inputs resident in HBM.  The patch matrix (265 MB) is
larger than L2, so no explicit flush is needed between steps; workloads
whose patch and residual matrices fit in L2 are timed step by step with an
L2 flush (a write larger than L2) before each step.

e2e = the same metric through the C ABI's ksvd_denoise with host buffers
(pinned): H2D of the image, patch gather, dictionary init, all iterations,
final OMP, image rebuild, D2H of the result, all inside the timed region;
value = patches x iterations / time per call.

Multi-GPU: the K-SVD iteration does not shard without a collective inside
the sequential atom sweep, so N GPUs run N independent replicas (each rank
its own seeded image): weak scaling, no data-path collective.

--impl reference times the CPU restatement of the reference's algorithm
(the reference has no CPU implementation of K-SVD) on the host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
from ksvd_loader import load, load_oracle  # noqa: E402

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def read_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return d, "measured"
        except Exception:
            pass
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def replica_workload(wl, rank):
    """Rank r denoises its own image: the workload with seed + r (replicas,
    no data exchanged between ranks)."""
    from dataclasses import replace
    return replace(wl, seed=wl.seed + rank)


def reduce_max(x, dist, device="cpu"):
    """Maximum of a per-rank float over all ranks (x itself without a group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, world, ms_max):
    """Whole-job rate: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / (ms_max / 1000.0)


def _cpu_sample_size(oracle, Y, D, wl, budget_s):
    """Patches per timed CPU iteration: the whole workload when one iteration
    is estimated to fit the budget, else a contiguous middle slice sized for it.
    The estimate separates the per-patch cost (OMP, Gram build) from the
    per-atom cost of the update (one n x n eigenproblem per atom)."""
    N = Y.shape[0]
    n1, n2 = min(N, 2048), min(N, 8192)
    times = []
    for ns in (n1, n2):
        Ys = np.ascontiguousarray(Y[(N - ns) // 2:(N - ns) // 2 + ns])
        t = time.perf_counter()
        idx, coef = oracle.omp(Ys, D, wl.omp_iter, dtype=np.float32)
        oracle.update_dictionary(Ys, D, idx, coef, q1_cap=False, dtype=np.float32)
        times.append(time.perf_counter() - t)
    per_patch = max((times[1] - times[0]) / max(n2 - n1, 1), 1e-9)
    fixed = max(times[0] - per_patch * n1, 0.0)
    if fixed + per_patch * N <= budget_s:
        return N
    return int(min(N, max(n2, (budget_s - fixed) / per_patch)))


def cpu_baseline(pkg, oracle, wl, budget_s=40.0):
    """One K-SVD iteration (FP32 OMP + full update sweep) of the CPU
    restatement, all host threads, on the whole workload if it fits the budget."""
    clean, noisy = wl.images()
    Y = oracle.extract_patches(noisy, wl.patch, wl.patch, wl.stride, wl.stride)
    N = Y.shape[0]
    D = oracle.init_dictionary(Y, wl.atoms, int_norm=True, dtype=np.float32)
    ns = _cpu_sample_size(oracle, Y, D, wl, budget_s)
    start = (N - ns) // 2
    Ys = np.ascontiguousarray(Y[start:start + ns])
    t = time.perf_counter()
    idx, coef = oracle.omp(Ys, D, wl.omp_iter, dtype=np.float32)
    oracle.update_dictionary(Ys, D, idx, coef, q1_cap=False, dtype=np.float32)
    dt = time.perf_counter() - t
    what = "all" if ns == N else f"a contiguous middle slice of {ns}"
    return {"value": ns / dt, "unit": "patches/s", "cores": oracle.max_threads(), "kind": "port",
            "sample": f"1 K-SVD iteration (FP32 OMP + full update sweep, {wl.atoms} atoms, L={wl.omp_iter}) on "
                      f"{what} of the workload's {N} patches, {dt:.1f} s"}, dt


def quality_vs_fp64(pkg, oracle, wl, clean, noisy, D0, patches, make_ctx, forms):
    """Accuracy of every form against the FP64 oracle on this workload (the
    checker, run after all timed regions): support agreement and coefficient
    error of the first OMP call from the shared initial dictionary, atom and
    coefficient error of the first update sweep from the FP64 codes, and the
    PSNR of the whole denoise beside the FP64 oracle's.  The oracle runs the
    same update mode as the timed steps (no 1024-patch cap)."""
    import torch
    import quality as q
    t0 = time.perf_counter()
    ref = q.fp64_reference(oracle, noisy, D0, patch=wl.patch, stride=wl.stride, omp_iter=wl.omp_iter,
                           ksvd_iter=wl.ksvd_iter, q1_cap=False, sigma2=wl.sigma ** 2)
    t_ref = time.perf_counter() - t0
    psnr64 = pkg.synth.psnr(clean, ref["image"])
    N, L = patches.shape[0], wl.omp_iter
    Dd = torch.from_numpy(D0).cuda()
    torch.cuda.synchronize()  # the contexts run on their own stream
    res = {"fp64_oracle_psnr": psnr64, "fp64_oracle_seconds": t_ref, "oracle_threads": oracle.max_threads(),
           "forms": {}}
    for form in forms:
        c, _ = make_ctx(form)
        idx = torch.empty((N, L), dtype=torch.int32, device="cuda")
        coef = torch.empty((N, L), dtype=torch.float32, device="cuda")
        c.omp(patches, Dd, idx, coef)
        torch.cuda.synchronize()
        i, cf = idx.cpu().numpy(), coef.cpu().numpy()
        out, _ = c.denoise(noisy, wl.sigma ** 2)
        p = pkg.synth.psnr(clean, out)
        res["forms"][form] = {"support_agreement": q.support_agreement(i, ref["idx0"]),
                              "coef_rel_err": q.coef_rel_err(i, cf, ref["idx0"], ref["coef0"]),
                              "psnr": p, "dpsnr_vs_fp64": p - psnr64}
        c.close()
    # the update sweep is shared by every form
    c, _ = make_ctx("fp32")
    D1 = torch.from_numpy(D0.copy()).cuda()
    idx = torch.from_numpy(ref["idx0"]).cuda()
    coef = torch.from_numpy(ref["coef0"].astype(np.float32)).cuda()
    torch.cuda.synchronize()
    c.update_dictionary(patches, D1, idx, coef)
    torch.cuda.synchronize()
    res["update_atom_err"] = q.atom_err(D1.cpu().numpy(), ref["D1"])
    res["update_coef_rel_err"] = q.coef_rel_err(ref["idx0"], coef.cpu().numpy(), ref["idx0"], ref["coef1"])
    c.close()
    res["bars"] = {"support_agreement": ">= 0.999", "coef_rel_err": "<= 1e-4", "update_atom_err": "<= 1e-4",
                   "dpsnr_vs_fp64": "|.| <= 0.05 dB"}
    return res


def batch_workload(pkg, ksvd, count=64, tune=False):
    """The uneven batch (64 seeded images, sides 256..2048, patches 8/12/22
    at stride 3, 16 speckle): ksvd_denoise_many end to end (host images in
    and out), beside the same images denoised one by one with ksvd_denoise in
    the same run.  Rate = patches x iterations / device time of the batch's
    iterations."""
    import torch
    jobs = pkg.synth.many_workload(count=count)
    specs = []
    for j in jobs:
        prm = ksvd.make_params(patch_width_dim=j["patch"], patch_height_dim=j["patch"], sliding_width=j["stride"],
                               sliding_height=j["stride"], atoms=j["atoms"], omp_iter=j["omp_iter"],
                               ksvd_iter=j["ksvd_iter"], speckle=int(j["speckle"]), compat=1,
                               precision=ksvd.PREC_FP16_RESCORE)
        specs.append((prm, j["noisy"], j["sigma2"]))
    ksvd.denoise_many(specs[:2], tune=False)  # warm-up (module load, first allocations)
    torch.cuda.synchronize()
    t = time.perf_counter()
    outs, st = ksvd.denoise_many(specs, tune=tune)
    wall_batch = time.perf_counter() - t
    t = time.perf_counter()
    seq_iter_ms = 0.0
    for prm, img, s2 in specs:
        with ksvd.Context(prm) as c:
            _, sst = c.denoise(img, s2)
            seq_iter_ms += sst["iter_ms"]
    wall_seq = time.perf_counter() - t
    T = jobs[0]["ksvd_iter"]
    psnr_gain = [pkg.synth.psnr(j["clean"], o) - pkg.synth.psnr(j["clean"], j["noisy"]) for j, o in zip(jobs, outs)]
    return {"images": count, "patches": st["num_patches"], "ksvd_iter": T,
            "sides": sorted({j["side"] for j in jobs}), "patch_sides": sorted({j["patch"] for j in jobs}),
            "speckle_images": sum(j["speckle"] for j in jobs),
            "iter_patches_per_s": st["num_patches"] * T / (st["iter_ms"] / 1000.0),
            "iter_ms": st["iter_ms"], "call_device_ms": st["total_ms"], "call_wall_s": wall_batch,
            "setup_ms": st["setup_ms"], "tune_ms": st["tune_ms"], "final_ms": st["final_ms"],
            "first_iter_codes_ms": st["codes_ms"], "first_iter_sweep_ms": st["sweep_ms"],
            "one_by_one_iter_ms": seq_iter_ms, "iter_speedup_vs_one_by_one": seq_iter_ms / st["iter_ms"],
            "one_by_one_wall_s": wall_seq, "wall_speedup_vs_one_by_one": wall_seq / wall_batch,
            "graph": st["graph"], "streams": st["streams"], "lanes": st["lanes"], "plan_ms": st["plan_ms"],
            "update_ctas_min_max": [min(st["update_ctas"]), max(st["update_ctas"])],
            "psnr_gain_db_min_median": [float(np.min(psnr_gain)), float(np.median(psnr_gain))],
            "form": "fp16 (tensor cores; 22x22 patches with the 16-bit dictionary streamed)"}


def workload_rates(pkg, ksvd, name, forms=("fp32", "fp16"), steps=3, warmup=1):
    """Patches/s per K-SVD iteration of another workload (device-timed K
    iterations from the initial dictionary after W warm-up ones), per form."""
    import torch
    wl = pkg.synth.WORKLOADS[name]
    _, noisy = wl.images()
    out = {"workload": name, "num_patches": wl.num_patches, "atoms": wl.atoms, "omp_iter": wl.omp_iter,
           "patch": f"{wl.patch}x{wl.patch}", "stride": wl.stride, "steps": steps, "warmup": warmup}
    precs = {"fp32": ksvd.PREC_FP32, "bf16": ksvd.PREC_BF16_RESCORE, "fp16": ksvd.PREC_FP16_RESCORE}
    patches = D = D0 = idx = coef = None
    for form in forms:
        params = ksvd.make_params(patch_width_dim=wl.patch, patch_height_dim=wl.patch, sliding_width=wl.stride,
                                  sliding_height=wl.stride, atoms=wl.atoms, omp_iter=wl.omp_iter, compat=1,
                                  precision=precs[form])
        with ksvd.Context(params) as c:
            c.set_stream(torch.cuda.current_stream().cuda_stream)  # the events below are on this stream
            if patches is None:
                N = ksvd.num_patches(params, wl.size, wl.size)
                patches = torch.empty((N, wl.n), dtype=torch.float32, device="cuda")
                D = torch.empty((wl.atoms, wl.n), dtype=torch.float32, device="cuda")
                idx = torch.empty((N, wl.omp_iter), dtype=torch.int32, device="cuda")
                coef = torch.empty((N, wl.omp_iter), dtype=torch.float32, device="cuda")
                c.extract_patches(torch.from_numpy(noisy).cuda(), patches)
                c.init_dictionary(patches, D)
                torch.cuda.synchronize()
                D0 = D.clone()
            D.copy_(D0)
            torch.cuda.synchronize()
            c.iterate(patches, D, idx, coef, warmup)
            D.copy_(D0)
            c.profile(1)
            c.profile_reset()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            c.iterate(patches, D, idx, coef, steps)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            fam = {f: c.profile_read(f)[0] / steps for f in ("gram", "omp", "csr", "residual", "update")}
            out[form] = {"patches_per_s": wl.num_patches / (ms / 1000.0), "ms_per_step": ms,
                         "kernel_ms_per_step": fam}
    del patches, D, D0, idx, coef
    torch.cuda.empty_cache()
    return out


def run_reference(args, wl):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    pkg = load()
    oracle = load_oracle()
    clean, noisy = wl.images()
    Y = oracle.extract_patches(noisy, wl.patch, wl.patch, wl.stride, wl.stride)
    N = Y.shape[0]
    D0 = oracle.init_dictionary(Y, wl.atoms, int_norm=True, dtype=np.float32)
    # each step sized so that warmup + steps fit in about three minutes
    steps_total = args.steps + args.warmup
    ns = _cpu_sample_size(oracle, Y, D0, wl, 180.0 / steps_total)
    start = (N - ns) // 2
    Ys = np.ascontiguousarray(Y[start:start + ns])
    D = D0.copy()
    times = []
    for i in range(steps_total):
        t = time.perf_counter()
        idx, coef = oracle.omp(Ys, D, wl.omp_iter, dtype=np.float32)
        D, coef = oracle.update_dictionary(Ys, D, idx, coef, q1_cap=False, dtype=np.float32)
        if i >= args.warmup:
            times.append(time.perf_counter() - t)
    ms = 1000.0 * float(np.mean(times))
    value = ns / (ms / 1000.0)
    cores = oracle.max_threads()
    line = {
        "metric": "patches/s per K-SVD iteration", "value": value, "unit": "patches/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl.name, "image": f"{wl.size}x{wl.size}", "sigma": wl.sigma,
                   "patch": f"{wl.patch}x{wl.patch}", "stride": wl.stride, "num_patches": N, "atoms": wl.atoms,
                   "omp_iter": wl.omp_iter, "sample_patches": ns},
        "cpu_baseline": {"value": value, "unit": "patches/s", "cores": cores, "kind": "port",
                         "sample": f"each step: 1 K-SVD iteration of the FP32 CPU restatement on "
                                   f"{'all' if ns == N else ns} of the workload's {N} patches, {cores} threads"},
        "e2e": {"value": value, "unit": "patches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="img2048_p12s3_k256")
    ap.add_argument("--precision", default="fp16", choices=["fp32", "bf16", "fp16", "learned"],
                    help="headline form; the other forms are timed beside it unless --no-forms")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--compat", type=int, default=1, help="KSVD_COMPAT_* bits (1 = INT_NORM, 3 = +Q1 cap)")
    ap.add_argument("--e2e-calls", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=40.0)
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-image uneven batch workload")
    ap.add_argument("--no-quality", action="store_true",
                    help="skip the accuracy report against the FP64 oracle (about a minute of CPU)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    pkg = load()
    wl = pkg.synth.WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference(args, wl)

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    ksvd = pkg.ksvd
    precs = {"fp32": ksvd.PREC_FP32, "bf16": ksvd.PREC_BF16_RESCORE, "fp16": ksvd.PREC_FP16_RESCORE,
             "learned": ksvd.PREC_BF16_LEARNED}
    learned = {}  # the fitted proposal (parameters, fit statistics), shared by the learned contexts

    def make_ctx(form):
        params = ksvd.make_params(patch_width_dim=wl.patch, patch_height_dim=wl.patch, sliding_width=wl.stride,
                                  sliding_height=wl.stride, atoms=wl.atoms, omp_iter=wl.omp_iter,
                                  ksvd_iter=wl.ksvd_iter, precision=precs[form], compat=args.compat, device=local)
        c = ksvd.Context(params)
        c.set_stream(stream.cuda_stream)
        if form == "learned":
            c.set_noise_variance(wl.sigma ** 2)
            if "params" in learned:
                c.proposal_set_params(learned["params"])
            else:
                # supports of ksvd_iter - 1 plain FP32 iterations from the
                # initial dictionary (about N x 9 pairs), 2 epochs
                st = c.proposal_fit(patches, D0, iters=max(1, wl.ksvd_iter - 1), epochs=2, seed=wl.seed)
                learned["params"] = c.proposal_get_params()
                learned["fit"] = st
        return c, params

    stream = torch.cuda.Stream()
    ctx, params = make_ctx("fp32" if args.precision == "learned" else args.precision)

    # each rank: its own seeded image (replicas)
    wlr = replica_workload(wl, rank)
    clean, noisy = wlr.images()
    H, W = noisy.shape
    N = ksvd.num_patches(params, W, H)
    n, K, L = wl.n, wl.atoms, wl.omp_iter
    sigma2 = wl.sigma ** 2

    with torch.cuda.stream(stream):
        img_d = torch.from_numpy(noisy).cuda()
        patches = torch.empty((N, n), dtype=torch.float32, device="cuda")
        D = torch.empty((K, n), dtype=torch.float32, device="cuda")
        idx = torch.empty((N, L), dtype=torch.int32, device="cuda")
        coef = torch.empty((N, L), dtype=torch.float32, device="cuda")
    stream.synchronize()
    ctx.extract_patches(img_d, patches)
    ctx.init_dictionary(patches, D)
    D0 = D.clone()
    if args.precision == "learned":
        ctx.close()
        ctx, params = make_ctx("learned")
    # the step's working set is the patch matrix plus the residual matrix of
    # the same size; below the L2 size (126 MB) steps are timed one by one
    # with an L2 flush between them
    l2_bytes = 126 * 1024 * 1024
    fits_l2 = 2 * N * n * 4 < l2_bytes
    flush_buf = None
    if fits_l2:
        with torch.cuda.stream(stream):
            flush_buf = torch.zeros(2 * l2_bytes // 4, dtype=torch.float32, device="cuda")
    stream.synchronize()

    def timed_steps(c, sample_clocks):
        """W warm-up iterations, then K timed ones from the initial dictionary.
        Returns (ms per step max over ranks, per-family ms, phases, counters,
        launches, clock summary)."""
        with torch.cuda.stream(stream):
            D.copy_(D0)
        for _ in range(args.warmup):
            c.iterate(patches, D, idx, coef, 1)
        stream.synchronize()
        with torch.cuda.stream(stream):
            D.copy_(D0)
        c.profile(1)
        c.profile_reset()
        l0 = c.launch_count()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps if flush_buf is not None else 1)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.__enter__()
        if flush_buf is None:
            evs[0][0].record(stream)
            for _ in range(args.steps):
                c.iterate(patches, D, idx, coef, 1)
            evs[0][1].record(stream)
        else:
            # inputs fit in L2: each step is timed alone, after a write of a
            # buffer larger than L2 (outside the step's events)
            for e0, e1 in evs:
                with torch.cuda.stream(stream):
                    flush_buf.add_(1)
                e0.record(stream)
                c.iterate(patches, D, idx, coef, 1)
                e1.record(stream)
        torch.cuda.synchronize()
        if sampler:
            sampler.__exit__(None, None, None)
        if dist:
            dist.barrier()
        ms = sum(e0.elapsed_time(e1) for e0, e1 in evs) / args.steps
        fams = {f: c.profile_read(f) for f in ("gram", "omp", "csr", "residual", "update", "proposal",
                                                "omp_restricted", "omp_fallback")}
        cn = c.profile_counters()
        # one more (untimed) iteration with the in-kernel phase timers on
        c.profile_reset()
        c.profile(2)
        c.iterate(patches, D, idx, coef, 1)
        ph = c.profile_phases()
        cn.update({k: v for k, v in c.profile_counters().items() if k.startswith("omp_")})
        c.profile(0)
        ms = reduce_max(ms, dist, "cuda")
        return ms, fams, ph, cn, c.launch_count() - l0, (sampler.summary() if sampler else None)

    # ---- the headline form: warm-up, then K timed K-SVD iterations ---------
    ms_step, fam, phases, counters, gpu_launches, clk_summary = timed_steps(ctx, True)
    value = aggregate_rate(N, world, ms_step)
    forms = {args.precision: value}
    fallback_rate = None
    if args.precision == "learned":
        fallback_rate = ctx.proposal_fallbacks()["last"] / N
    if not args.no_forms:
        for form in ("fp32", "fp16", "bf16", "learned"):
            if form == args.precision:
                continue
            c2, _ = make_ctx(form)
            ms2 = timed_steps(c2, False)[0]
            forms[form] = aggregate_rate(N, world, ms2)
            if form == "learned":
                fallback_rate = c2.proposal_fallbacks()["last"] / N
            c2.close()

    # ---- e2e through the C ABI with pinned host buffers --------------------
    img_h = torch.from_numpy(noisy).pin_memory()
    out_h = torch.empty_like(img_h).pin_memory()
    e2e_ms = []
    st = None
    for i in range(max(args.e2e_calls, 1) + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = ctx.denoise_ptr(img_h.data_ptr(), W, H, sigma2, out_h.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        if i > 0:  # first call is a warm-up
            e2e_ms.append(e0.elapsed_time(e1))
    # one more call with per-family timing: the gather and the rebuild
    ctx.profile(1)
    ctx.profile_reset()
    ctx.denoise_ptr(img_h.data_ptr(), W, H, sigma2, out_h.data_ptr())
    img_fams = {f: ctx.profile_read(f) for f in ("im2col", "col2im", "blend")}
    ctx.profile(0)
    e2e_call_ms = float(np.median(e2e_ms))
    e2e_call_ms = reduce_max(e2e_call_ms, dist, "cuda")
    e2e_value = aggregate_rate(N * wl.ksvd_iter, world, e2e_call_ms)
    out = out_h.numpy()
    psnr_noisy = pkg.synth.psnr(clean, noisy)
    psnr_out = pkg.synth.psnr(clean, out)

    if rank == 0:
        peaks, peak_src = read_peaks()
        # dominant kernel by device time
        dom = max(("omp", "update"), key=lambda f: fam[f][0])
        dom_ms, dom_launches = fam[dom]
        avg_ms = dom_ms / max(dom_launches, 1)
        # algorithmic bytes per launch, per patch times the patches of a launch:
        #   omp: read the patch (4n) + write the codes (8L)
        #   update: read the patch once per used atom + code (L(4n+8)) + write coefficients (4L)
        # (the 16-bit forms' OMP also writes the sweep's residual rows, 4n
        # more, when no separate residual pass ran)
        omp_bpp = 4 * n + 8 * L + (4 * n if fam["residual"][0] <= 0.0 else 0)
        if dom == "omp":
            bytes_per_patch = omp_bpp
        else:
            bytes_per_patch = L * (4 * n + 8) + 4 * L
        traffic_file = ROOT / "profiles" / f"traffic_{wl.name}_{args.precision}.json"
        traffic = None
        if traffic_file.exists():
            try:
                traffic = json.loads(traffic_file.read_text()).get(dom)
            except Exception:
                traffic = None
        achieved = bytes_per_patch * N / (avg_ms / 1000.0) / 1e9
        peak = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
        peak_tc = float(peaks.get("bf16_tflops", PEAKS_FALLBACK["bf16_tflops"]))
        # every kernel family against its own bound (algorithmic work per
        # patch x patches / device time per step); the correlation of the
        # 16-bit forms against the tensor peak, the rest against HBM
        flops_pp = 2 * n * K * L
        per_kernel = {}
        for f, bpp in (("omp", omp_bpp), ("update", L * (4 * n + 8) + 4 * L), ("residual", 8 * n + 8 * L),
                       ("csr", 12 * L)):
            ms_f = fam[f][0] / max(args.steps, 1)
            if ms_f <= 0:
                continue
            gbs = bpp * N / (ms_f / 1000.0) / 1e9
            per_kernel[f] = {"ms_per_step": ms_f, "bytes_per_patch": bpp, "achieved_gbs": gbs,
                             "frac_hbm": gbs / peak}
            if f == "omp" and args.precision != "fp32":
                tfs = flops_pp * N / (ms_f / 1000.0) / 1e12
                per_kernel[f].update({"flops_per_patch": flops_pp, "achieved_tflops": tfs,
                                      "frac_tensor": tfs / peak_tc})
        # the patch gather and the image rebuild (per call of ksvd_denoise):
        #   im2col: write the patches (4n per patch) + read the image (4 per pixel)
        #   col2im: read the codes (8L per patch) + read the noisy image and
        #           write the overlap sums (8 per pixel); the dictionary is L2-resident
        for f, nbytes in (("im2col", 4 * n * N + 4 * W * H), ("col2im", 8 * L * N + 8 * W * H)):
            ms_f = img_fams[f][0]
            if ms_f > 0:
                gbs = nbytes / (ms_f / 1000.0) / 1e9
                per_kernel[f] = {"ms_per_call": ms_f, "bytes_per_call": nbytes, "achieved_gbs": gbs,
                                 "frac_hbm": gbs / peak}
        # the whole iteration against max(F / tensor peak, B / HBM peak) with
        # the compulsory bytes B = 4n + 8L (OMP) + L(4n + 8) + 4L (update)
        b_iter = 4 * n + 8 * L + L * (4 * n + 8) + 4 * L
        t_bound = max(flops_pp * N / (peak_tc * 1e12), b_iter * N / (peak * 1e9))
        iter_bound = {"bytes_per_patch": b_iter, "flops_per_patch": flops_pp,
                      "bound_patches_per_s": N / t_bound, "frac": (value / world) / (N / t_bound)}
        cpu = None
        if not args.no_cpu_baseline:
            oracle = load_oracle()
            cpu, _ = cpu_baseline(pkg, oracle, wl, budget_s=args.cpu_budget)
        batch = big = None
        if not args.no_batch and world == 1:
            batch = batch_workload(pkg, ksvd)
            big = workload_rates(pkg, ksvd, "img4096_p16s2_k512", forms=("fp32", "fp16", "bf16"))
        acc = None
        if not args.no_quality and world == 1:
            acc = quality_vs_fp64(pkg, load_oracle(), wl, clean, noisy, D0.cpu().numpy(), patches, make_ctx,
                                  list(forms))
        # the metric by form: patches/s per iteration, ratio over the plain
        # FP32 form, and the accuracy beside it
        by_form = {}
        for f, v in forms.items():
            by_form[f] = {"patches_per_s": v, "ratio_vs_fp32": (v / forms["fp32"]) if "fp32" in forms else None}
            if acc:
                by_form[f].update(acc["forms"][f])
        if "learned" in by_form:
            by_form["learned"]["fallback_rate_last_step"] = fallback_rate
            by_form["learned"]["fit"] = learned.get("fit")
            by_form["learned"]["note"] = ("proposal fitted before timing on this image's own plain-FP32 supports "
                                          "(ksvd_iter - 1 iterations, 2 epochs); fit time not in the metric")
        line = {
            "metric": "patches/s per K-SVD iteration", "value": value, "unit": "patches/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp32": "f32", "bf16": "bf16+f32+f64", "fp16": "f16+f32+f64",
                      "learned": "bf16+f32+f64"}[args.precision],
            "data": "synthetic",
            "config": {"workload": wl.name, "image": f"{wl.size}x{wl.size}", "sigma": wl.sigma,
                       "patch": f"{wl.patch}x{wl.patch}", "stride": wl.stride, "num_patches": N, "atoms": K,
                       "omp_iter": L, "precision": args.precision, "compat": args.compat,
                       "l2": (f"inputs fit in L2 ({N * n * 4 / 1e6:.0f} MB patch matrix): L2 flushed before "
                              f"each step by a {2 * l2_bytes / 1e6:.0f} MB write, steps timed one by one"
                              if fits_l2 else
                              f"inputs larger than L2 ({N * n * 4 / 1e6:.0f} MB patch matrix), no flush"),
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_value, "unit": "patches/s", "h2d_bytes_per_step": int(W * H * 4),
                    "d2h_bytes_per_step": int(W * H * 4), "ms_per_call": e2e_call_ms,
                    "ksvd_iter_per_call": wl.ksvd_iter},
            "gpu_launches": int(gpu_launches),
            "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "algorithmic_bytes_per_patch": bytes_per_patch, "avg_launch_ms": avg_ms},
            "kernel_ms_per_step": {f: fam[f][0] / max(args.steps, 1) for f in fam},
            "roofline_per_kernel": per_kernel,
            "iteration_vs_bound": iter_bound,
            "phase_ms_one_step": {
                name: phases[i] for i, name in (
                    (7, "upd_setup"), (0, "upd_wait_prev_atom"), (1, "upd_load"), (2, "upd_pass"),
                    (3, "upd_wait_partials"), (4, "upd_allreduce"), (5, "upd_coef_store"), (8, "omp_corr"),
                    (9, "omp_residual"), (10, "omp_io"), (11, "omp_rescore"), (12, "omp_cholesky"))},
            "counters_per_step": {k: (v if k.startswith("omp_") else v / max(args.steps, 1))
                                  for k, v in counters.items()},
            "quality": {"psnr_noisy": psnr_noisy, "psnr_denoised": psnr_out,
                        "power_iters_last_sweep": st.power_iters, "atoms_updated_last_sweep": st.atoms_updated,
                        "vs_fp64_oracle": acc},
            "forms_patches_per_s": forms,
            "metric_by_form": by_form,
            "extra_workloads": {"batch64_uneven": batch, "img4096_p16s2_k512": big},
            "clocks": clk_summary,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
