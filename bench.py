#!/usr/bin/env python
"""Benchmark: OSEM sub-iteration of FIR's clinical configuration on B200.

A step is one OSEM sub-iteration (reconAlgos.cc:119-198) of the clinical
workload: 32 rings x 512 crystals, R = 400 mm, LORs within a 300 mm FOV
(3.28e7 LORs, 16 subsets of 2.05e6), 200x200x64 image at 3 mm, FWHM 4 mm
Gaussian filter every sub-iteration, seeded synthetic phantom with water
attenuation and 5e8 Poisson counts.  The metric counts ray-voxel steps the
way FIR enumerates them: every path element of every LOR of the subset for
the projection, plus every path element of the LORs whose estimate exceeds
1e-5 for the backprojection.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fir|reference]

Prints one JSON line (rank 0).  --impl reference times FIR's own OpenMP code
(compiled from its sources into oracle/_ref) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ray-voxel steps/s fwd+bck; OSEM s/iter; batched & plain GPU vs CPU at ≤1e-4 err"
UNIT = "ray-voxel steps/s"
EPS = 1e-5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=32)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", choices=["fir", "reference"], default="fir")
    ap.add_argument("--workload", choices=["clinical", "small", "large"], default="clinical")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-runs", type=int, default=3, help="timed fir_osem calls of the e2e leg (median)")
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--det-steps", type=int, default=2,
                    help="extra sub-iterations timed with deterministic backprojection (0: skip)")
    ap.add_argument("--float-steps", type=int, default=8,
                    help="extra sub-iterations timed with the opt-in float traversal (0: skip)")
    ap.add_argument("--skip-zero-steps", type=int, default=4,
                    help="extra sub-iterations timed with FIR_OPT_SKIP_ZERO_BINS (0: skip)")
    ap.add_argument("--batch-runs", type=int, default=2,
                    help="timed runs of the 64-problem batched OSEM and of its sequential plain form (0: skip)")
    ap.add_argument("--batch-problems", type=int, default=64)
    ap.add_argument("--large-runs", type=int, default=2,
                    help="timed OSEM iterations of the large workload, plain and as one graph (0: skip)")
    ap.add_argument("--lbfgs-steps", type=int, default=50,
                    help="L-BFGS iterations of the differentiable-projector section (0: skip the section)")
    return ap.parse_args()


def workload(name):
    from fir_b200 import workloads

    return {"clinical": workloads.clinical, "small": workloads.small, "large": workloads.large}[name]()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """Per-launch DRAM bytes of the OSEM kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "osem_subset_clinical.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# -------------------------------------------------------------- step counts

def subset_of_bins(proj, n_subsets, torch, device):
    """Subset index (view % n_subsets) of every bin, flat file order."""
    from fir_b200 import capi

    g = capi.proj_geometry(proj)
    parts = []
    for nax in g["n_axial"]:
        bpv = nax * g["n_tang_coords"]
        v = torch.arange(g["n_views"], device=device, dtype=torch.int32).repeat_interleave(bpv)
        parts.append(v % n_subsets)
    return torch.cat(parts)


def reference_counts(w, ref, n_bins, cache_dir="/tmp"):
    """Path elements per bin by FIR's own Siddon (oracle/_ref, all threads)."""
    import numpy as np

    key = f"{w.name}_{w.proj.n_rings}_{w.proj.n_crystals_per_ring}_{w.proj.n_tang_coords}_{w.vol.size[0]}"
    path = os.path.join(cache_dir, f"fir_counts_{key}.npy")
    if os.path.exists(path):
        c = np.load(path)
        if c.size == n_bins:
            return c
    c = ref.path_counts(w.scanner, w.proj, w.vol, n_bins)
    try:
        np.save(path, c)
    except Exception:
        pass
    return c


def bench_config(w, world, n_bins):
    """The `config` object of the JSON line, the same for both arms."""
    nsub = w.osem.n_subsets
    return {
        "workload": f"{w.name}: OSEM sub-iteration, {w.proj.n_rings} rings x {w.proj.n_crystals_per_ring} "
                    f"crystals, {w.proj.n_tang_coords} tangential bins, {n_bins} LORs, "
                    f"{'x'.join(str(s) for s in w.vol.size)} @ {w.vol.voxel[0]} mm, {nsub} subsets, "
                    f"FWHM {w.osem.fwhm_xyz[0]} mm, seeded phantom, water attenuation, "
                    f"{w.counts:.0e} Poisson counts",
        "l2": "flushed (256 MB write) before every timed step, outside the step's events",
        "parallelism": f"views of each subset split over {world} GPUs, NCCL all-reduce of the backprojection"
                       if world > 1 else "single GPU",
    }


# ------------------------------------------------------------ CPU reference

def reference_inputs(w, ref):
    """The benchmark's measured data and sensitivity made by FIR's own
    compiled code (oracle/_ref): HU-to-mu map, forward projections of the
    mu map and of the phantom, and the subsets' sensitivity.  The sinogram
    is bit-identical to the GPU arm's (both forward projectors are
    bit-identical to FIR and the rest is workloads.measured_sinogram)."""
    from fir_b200 import workloads

    nb = ref.proj_geometry(w.proj)["n_bins"]
    mu = ref.hu_to_mu(w.vol, workloads.hounsfield(w))
    line_mu = ref.forward(w.scanner, w.proj, w.vol, mu, nb)
    ax = ref.forward(w.scanner, w.proj, w.vol, workloads.activity(w), nb)
    y = workloads.measured_sinogram(w, ax, line_mu)
    sens = ref.sensitivity(w.scanner, w.proj, w.vol, w.osem.n_subsets)
    return nb, y, sens


def cpu_reference_run(w, ref, y, sens, img0, counts, iters):
    """Times FIR's reconAlgos::OSEM (oracle/_ref, all host threads) for
    `iters` full iterations of the workload on the given data, sensitivity
    and start image.  Steps are counted as FIR enumerates them: every path
    element of every LOR for the projection, and for the backprojection
    every element of every crossing LOR (exact from a uniform start image,
    where every crossing LOR's estimate is positive; an upper bound after
    that, which favours FIR)."""
    import numpy as np

    from fir_b200.geometry import OSEMParams

    cores = os.cpu_count() or 1
    ref.threads(cores)
    nsub = w.osem.n_subsets
    img = np.ascontiguousarray(img0, np.float32)
    prm = OSEMParams(n_iterations=1, n_subsets=nsub, convolution_interval=w.osem.convolution_interval,
                     fwhm_xyz=list(w.osem.fwhm_xyz), cut_radius=w.osem.cut_radius)
    t0 = time.perf_counter()
    for _ in range(iters):
        img = ref.osem(w.scanner, w.proj, w.vol, y, img, sens, prm)
    dt = time.perf_counter() - t0
    steps = 2 * int(counts.sum(dtype=np.int64)) * iters
    return {
        "value": steps / dt,
        "unit": UNIT,
        "cores": cores,
        "kind": "reference",
        "seconds": dt,
        "osem_s_per_iteration": dt / iters,
        "sample": f"{iters} full OSEM iteration(s) of the {w.name} workload ({nsub} sub-iterations each) by "
                  f"FIR's reconAlgos::OSEM compiled -O3 -fopenmp, {cores} threads, on the same measured data "
                  f"and sensitivity as the GPU arm; S = {steps} ray-voxel steps",
    }


def reference_arm(args, rank):
    """FIR's own OpenMP implementation of the path (oracle/_ref), on the host
    cores, on the GPU arm's workload, data and config.  Nothing of fir_b200's
    native library is loaded in this process."""
    if rank != 0:
        return 0
    w = workload(args.workload)
    try:
        from oracle import bridge

        if not bridge.reference_available():
            raise FileNotFoundError("oracle/_ref/libfirref.so not built")
        ref = bridge.Reference()
    except Exception as e:  # noqa: BLE001
        print(json.dumps({"impl": "reference", "unavailable": f"FIR reference library unavailable: {e}"}))
        return 0
    import numpy as np

    world = int(os.environ.get("WORLD_SIZE", "1"))
    ref.threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    nb, y, sens = reference_inputs(w, ref)
    counts = reference_counts(w, ref, nb)
    prep_s = time.perf_counter() - t0
    nsub = w.osem.n_subsets
    budget = max(nsub, min(args.steps, 2 * nsub))
    iters = max(1, int(math.ceil(budget / nsub)))
    r = cpu_reference_run(w, ref, y, sens, np.ones(w.vol.shape_zyx, np.float32), counts, iters)
    ms = 1000.0 * r["osem_s_per_iteration"] / nsub
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": r["value"],
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32 data, f64 geometry",
        "data": "synthetic (seeded phantom, water attenuation, Poisson counts)",
        "config": bench_config(w, world, nb),
        "osem_s_per_iteration": r["osem_s_per_iteration"],
        "input_prep_s": prep_s,
        "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------ the GPU arm

def path_steps(ctx, w, torch, dev):
    """Traversal steps of every LOR of w (our traversal; bookkeeping)."""
    import ctypes as C

    from fir_b200 import capi

    nb = w.n_lors
    counts = torch.empty(nb, dtype=torch.int32, device=dev)
    crosses = torch.empty(nb, dtype=torch.int32, device=dev)
    bins = torch.arange(nb, dtype=torch.int64, device=dev)
    ctx.use_torch_stream()
    capi._check(capi.lib().fir_lor_paths(ctx.handle, C.byref(capi.proj_desc(w.proj)),
                                         C.byref(capi.vol_desc(w.vol, 1)), nb, bins.data_ptr(), 0, None, None,
                                         counts.data_ptr(), crosses.data_ptr()))
    return int(counts.to(torch.int64).sum())


def batched_section(args, local):
    """64 independent reconstructions of uneven sizes: one batched schedule
    (persistent projector, autotuned launch shape, CUDA graph) against the
    same problems run one after another through fir_osem."""
    import numpy as np
    import torch

    from fir_b200 import capi, workloads

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    ws = workloads.batch_problems(args.batch_problems)
    ctx = capi.Context(device=local)
    data, steps = [], 0
    for w in ws:
        ctx.set_scanner(w.scanner)
        y, sens = workloads.measured_on_gpu(ctx, w, dev, attenuation=False)
        data.append((y, sens))
        # fwd + back steps: both traversals of every LOR, once per iteration
        steps += 2 * w.osem.n_iterations * path_steps(ctx, w, torch, dev)
    torch.cuda.synchronize()

    def timed(fn, before=None):
        out = []
        for _ in range(args.batch_runs):
            if before is not None:
                before()
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            out.append(a.elapsed_time(b))
        return out

    # sequential plain form: one context per problem, created beforehand
    plain_ctx = [capi.Context(w.scanner, device=local) for w in ws]
    imgs = [torch.ones(w.vol.shape_zyx, device=dev) for w in ws]

    def reset_plain():
        for im in imgs:
            im.fill_(1.0)

    def run_plain():
        for c, w, (y, sens), im in zip(plain_ctx, ws, data, imgs):
            c.osem(w.proj, y, w.vol, im, sens, w.osem)

    reset_plain()
    run_plain()  # warm: scratch allocation
    l0 = sum(c.launch_count for c in plain_ctx)
    plain_ms = timed(run_plain, reset_plain)
    plain_launches = (sum(c.launch_count for c in plain_ctx) - l0) // args.batch_runs

    ctx.use_torch_stream()
    batch = capi.Batch(ctx, [(w.scanner, w.proj, w.vol, w.osem) for w in ws])
    ones = [np.ones(w.vol.shape_zyx, np.float32) for w in ws]

    def reset_batch():
        for k in range(len(ws)):
            batch.set_image(k, ones[k])

    for k, (y, sens) in enumerate(data):
        batch.set_data(k, y, sens)
    reset_batch()
    t0 = time.perf_counter()
    tune_ms = batch.tune()
    tune_wall = time.perf_counter() - t0
    tune_table = batch.tune_report()
    shape = batch.launch()
    n_steps, launches = batch.schedule()
    batch.osem(use_graph=True)  # warm: capture + instantiate
    graph_ms = timed(lambda: batch.osem(use_graph=True), reset_batch)
    direct_ms = timed(lambda: batch.osem(use_graph=False), reset_batch)
    reset_batch()
    batch.osem(use_graph=True)
    err = 0.0
    for k in range(len(ws)):
        got = batch.get_image(k)
        want = imgs[k].cpu().numpy()
        err = max(err, float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30)))
    axial_tile = batch.bundle()
    batch.close()
    for c in plain_ctx:
        c.close()
    ctx.close()
    g, p, d = min(graph_ms), min(plain_ms), min(direct_ms)
    return {
        "value": steps / (g / 1000.0),
        "unit": UNIT,
        "plain_value": steps / (p / 1000.0),
        "speedup_vs_plain": p / g,
        "ms_batched_graph": g,
        "ms_batched_direct": d,
        "ms_plain_sequential": p,
        "problems": len(ws),
        "lors": int(sum(w.n_lors for w in ws)),
        "voxels": int(sum(w.vol.n_voxels for w in ws)),
        "schedule_steps": n_steps,
        "gpu_launches": launches,
        "plain_gpu_launches": plain_launches,
        "launch_shape": {"block": shape[0], "blocks_per_sm": shape[1], "grab": shape[2],
                         "axial_tile": axial_tile},
        "tuner_best_step0_ms": tune_ms,
        "tuner_candidates": [{"block": b, "blocks_per_sm": p, "grab": gr, "axial_tile": at, "step0_ms": round(t, 4)}
                             for b, p, gr, at, t in tune_table],
        "tuner_wall_s": tune_wall,
        "max_rel_l2_vs_plain": err,
        "runs": args.batch_runs,
        "workload": "64 seeded problems: 4-24 rings x 96-384 crystals, R 150-400 mm, images 32^2x8..128^2x48 "
                    "at 2-4 mm, cylinder + 2 spheres, 1e5-1e7 Poisson counts, 4-12 subsets x 3 iterations, "
                    "FWHM 4 mm; whole OSEM of all problems per run (best of runs)",
        "steps_counted": "2 x path steps of every LOR per iteration (forward and back traversal), same count "
                         "for both forms",
    }


def autograd_section(args, local):
    """Differentiable projector on the clinical scanner: 8 ellipsoid phantoms
    (128x128x48 at 3 mm) with water attenuation and Poisson data; penalized
    Poisson NLL (beta = 0.01, quadratic 26-neighbour); gradient time, adjoint
    test and an L-BFGS reconstruction."""
    import numpy as np
    import torch

    from fir_b200 import autograd as fa
    from fir_b200 import workloads

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    ws = workloads.autograd_batch(8)
    w0 = ws[0]
    op = fa.SiddonProjector(w0.scanner, w0.proj, w0.vol, device=local)
    nb = op.n_bins
    mu = torch.stack([torch.from_numpy(workloads.hounsfield(w)) for w in ws]).to(dev)
    x_true = torch.stack([torch.from_numpy(workloads.activity(w)) for w in ws]).to(dev)
    for f in range(len(ws)):
        op.ctx.hu_to_mu(w0.vol, mu[f])
    atten = torch.exp(-op.project(mu))  # exp(-A mu) per frame
    ybar = op.project(x_true) * atten
    ybar *= (w0.counts / ybar.sum(dim=1, dtype=torch.float64)).float()[:, None]
    scale = (w0.counts / (op.project(x_true) * atten).sum(dim=1, dtype=torch.float64)).float()[:, None]
    atten = atten * scale
    y = torch.poisson(ybar, generator=torch.Generator(device=dev).manual_seed(w0.seed))
    del ybar, mu
    steps_per_frame = path_steps(op.ctx, w0, torch, dev)
    beta = 0.01

    # adjoint test on random non-negative x, y
    g = torch.Generator(device=dev).manual_seed(9)
    xr = torch.rand(x_true.shape, generator=g, device=dev)
    yr = torch.rand(y.shape, generator=g, device=dev)
    lhs = float((op.project(xr).double() * yr.double()).sum())
    rhs = float((xr.double() * op.backproject(yr).double()).sum())
    del xr, yr

    # time per gradient: forward projection of 8 frames, loss, backprojection
    x = torch.ones_like(x_true).requires_grad_(True)
    times = []
    for i in range(3 + 5):
        x.grad = None
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        loss = fa.penalized_nll(x, y, op, beta, atten)
        loss.backward()
        b.record(stream)
        torch.cuda.synchronize()
        if i >= 3:
            times.append(a.elapsed_time(b))
    grad_ms = sum(times) / len(times)
    # central finite differences (h = 1e-3, float64) of the first phantom's
    # penalized NLL at 64 random voxels inside the field of view
    a64, y64 = atten[:1].double(), y[:1].double()
    xd = (0.5 + 0.5 * torch.rand((1,) + tuple(w0.vol.shape_zyx), generator=g, device=dev,
                                 dtype=torch.float64)).requires_grad_(True)
    fa.penalized_nll(xd, y64, op, beta, a64).backward()
    gd = xd.grad.detach()
    rng = np.random.default_rng(16)
    nz, ny, nx = w0.vol.shape_zyx
    fd_worst, h = 0.0, 1e-3
    with torch.no_grad():
        for _ in range(64):
            while True:
                j = (0, int(rng.integers(nz)), int(rng.integers(ny)), int(rng.integers(nx)))
                if (j[2] - ny / 2) ** 2 + (j[3] - nx / 2) ** 2 < 45 ** 2:
                    break
            xp, xm = xd.detach().clone(), xd.detach().clone()
            xp[j] += h
            xm[j] -= h
            # the loss difference summed bin by bin: the totals (~1e9) would
            # carry rounding errors of ~1e-6 each
            tp = fa.expected_counts(xp, op, a64)
            tm = fa.expected_counts(xm, op, a64)
            dl = float(((tp - torch.xlogy(y64, tp)) - (tm - torch.xlogy(y64, tm))).sum())
            dl += float(fa.quadratic_penalty(xp, beta) - fa.quadratic_penalty(xm, beta))
            fd = dl / (2 * h)
            fd_worst = max(fd_worst, abs(fd - float(gd[j])) / max(abs(float(gd[j])), 1e-3))
    del xd, gd, a64, y64

    launches0 = op.ctx.launch_count
    xr, stats = fa.reconstruct_lbfgs(op, y, beta, atten, steps=args.lbfgs_steps)
    launches = op.ctx.launch_count - launches0
    corr = float(np.corrcoef(xr.cpu().numpy().ravel(), x_true.cpu().numpy().ravel())[0, 1])
    op.close()
    n = len(ws)
    return {
        "ms_per_gradient": grad_ms,
        "value": 2 * n * steps_per_frame / (grad_ms / 1000.0),
        "unit": UNIT,
        "steps_counted": "forward and back traversal of every LOR, per frame",
        "traversal_value": 2 * math.ceil(n / 4) * steps_per_frame / (grad_ms / 1000.0),
        "traversal_steps_counted": "forward and back traversal of every LOR per group of up to 4 frames (one "
                                   "traversal serves 4 frames): comparable with the plain sub-iteration's rate",
        "frames": n,
        "lors_per_frame": nb,
        "adjoint_rel_error": abs(lhs - rhs) / abs(lhs),
        "finite_difference_max_rel_error": fd_worst,
        "finite_difference": "central, h = 1e-3, float64, 64 random voxels of the first phantom inside the FOV",
        "lbfgs_steps": args.lbfgs_steps,
        "lbfgs_evaluations": stats["evaluations"],
        "lbfgs_ms_per_gradient": sum(stats["gradient_ms"]) / max(1, len(stats["gradient_ms"])),
        "lbfgs_wall_s": stats["wall_s"],
        "lbfgs_loss_first_last": [stats["losses"][0], stats["losses"][-1]],
        "lbfgs_projector_launches": launches,
        "recon_corr_with_phantom": corr,
        "workload": "clinical scanner (32 rings x 512 crystals, 125 tangential bins), 8 seeded ellipsoid phantoms "
                    "128x128x48 @ 3 mm, water attenuation, 5e8 Poisson counts each; loss = Poisson NLL + "
                    "0.01 x quadratic 26-neighbour penalty; float32",
    }


def large_section(args, local):
    """The large workload: one OSEM iteration (all subsets) through fir_osem,
    and the same iteration captured as one CUDA graph (a batch of one
    problem, autotuned)."""
    import numpy as np
    import torch

    from fir_b200 import capi, workloads

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    w = workloads.large()
    ctx = capi.Context(w.scanner, device=local)
    ctx.set_option(capi.FIR_OPT_GEOMETRY, w.geometry)
    y, sens = workloads.measured_on_gpu(ctx, w, dev, attenuation=True)
    steps = 2 * w.osem.n_iterations * path_steps(ctx, w, torch, dev)
    img = torch.ones(w.vol.shape_zyx, device=dev)
    ctx.osem(w.proj, y, w.vol, img, sens, w.osem)  # warm
    plain = []
    for _ in range(args.large_runs):
        img.fill_(1.0)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.osem(w.proj, y, w.vol, img, sens, w.osem)
        b.record(stream)
        torch.cuda.synchronize()
        plain.append(a.elapsed_time(b))
    batch = capi.Batch(ctx, [(w.scanner, w.proj, w.vol, w.osem)])
    batch.set_data(0, y, sens)
    ones = np.ones(w.vol.shape_zyx, np.float32)
    batch.set_image(0, ones)
    batch.tune()
    shape = batch.launch()
    n_steps, launches = batch.schedule()
    batch.osem(use_graph=True)  # capture
    graph = []
    for _ in range(args.large_runs):
        batch.set_image(0, ones)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        batch.osem(use_graph=True)
        b.record(stream)
        torch.cuda.synchronize()
        graph.append(a.elapsed_time(b))
    got = batch.get_image(0)
    want = img.cpu().numpy()
    err = float(np.linalg.norm(got - want) / np.linalg.norm(want))
    batch.close()
    ctx.close()
    p, g = min(plain), min(graph)
    return {
        "value": steps / (g / 1000.0),
        "unit": UNIT,
        "plain_value": steps / (p / 1000.0),
        "osem_s_per_iteration_graph": g / 1000.0,
        "osem_s_per_iteration_plain": p / 1000.0,
        "subsets": w.osem.n_subsets,
        "lors": w.n_lors,
        "graph_launches": launches,
        "launch_shape": {"block": shape[0], "blocks_per_sm": shape[1], "grab": shape[2]},
        "rel_l2_graph_vs_plain": err,
        "steps_counted": "2 x path steps of every LOR per iteration",
        "workload": "64 rings x 640 crystals, R 410 mm, pitch 3.2 mm, 163 tangential bins (160 mm FOV), "
                    "320x320x128 @ 1.5 mm (exact geometry), 40 ellipsoids + 20 hot spheres, water attenuation, "
                    "2e9 Poisson counts, 32 subsets x 1 iteration, FWHM 4 mm; best of runs",
    }


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return reference_arm(args, rank)

    import numpy as np
    import torch

    from fir_b200 import capi, workloads

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    w = workload(args.workload)
    nsub = w.osem.n_subsets
    nb = w.n_lors
    nvox = w.vol.n_voxels
    ctx = capi.Context(w.scanner, device=local)
    aux = capi.Context(w.scanner, device=local)  # bookkeeping (untimed)
    if w.geometry:
        ctx.set_option(capi.FIR_OPT_GEOMETRY, w.geometry)
        aux.set_option(capi.FIR_OPT_GEOMETRY, w.geometry)
    if args.block:
        ctx.set_option(capi.FIR_OPT_BLOCK_SIZE, args.block)

    # ---- data: attenuated, scaled, Poisson-sampled, precorrected (OSEM.cc:294-337);
    # the two forward projections are bit-identical to FIR's, and the rest is
    # host numpy, so the reference arm builds the same sinogram with FIR
    x_true = torch.from_numpy(workloads.activity(w)).to(dev)
    mu = torch.from_numpy(workloads.hounsfield(w)).to(dev)
    aux.hu_to_mu(w.vol, mu)
    line_mu = torch.empty(nb, device=dev)
    aux.forward(w.vol, mu, w.proj, line_mu)
    ax = torch.empty(nb, device=dev)
    aux.forward(w.vol, x_true, w.proj, ax)
    y_host = workloads.measured_sinogram(w, ax.cpu().numpy(), line_mu.cpu().numpy())
    y = torch.from_numpy(y_host).to(dev)
    del ax, x_true, line_mu, mu
    sens = torch.empty((nsub,) + tuple(w.vol.shape_zyx), device=dev)
    aux.sensitivity(w.proj, w.vol, sens, nsub)
    img = torch.ones(w.vol.shape_zyx, device=dev)
    sens_frames = [sens[s] for s in range(nsub)]

    # path elements of every bin, by our own traversal (bookkeeping)
    counts = torch.empty(nb, dtype=torch.int32, device=dev)
    crosses = torch.empty(nb, dtype=torch.int32, device=dev)
    bins = torch.arange(nb, dtype=torch.int64, device=dev)
    import ctypes as C

    aux.use_torch_stream()
    capi._check(capi.lib().fir_lor_paths(aux.handle, C.byref(capi.proj_desc(w.proj)), C.byref(capi.vol_desc(w.vol, 1)),
                                         nb, bins.data_ptr(), 0, None, None, counts.data_ptr(), crosses.data_ptr()))
    del bins
    subset_id = subset_of_bins(w.proj, nsub, torch, dev)
    counts64 = counts.to(torch.int64)
    s_fwd = [int(counts64[subset_id == s].sum()) for s in range(nsub)]
    line = torch.empty(nb, device=dev)

    def s_bwd(subset):
        aux.forward(w.vol, img, w.proj, line)
        m = (subset_id == subset) & (line.double() > EPS)
        return int(counts64[m].sum())

    prm = w.osem
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    # One step = one sub-iteration of the whole job.  On N GPUs each rank
    # backprojects 1/N of the subset's views and one NCCL all-reduce sums the
    # backprojection (fir_b200.distributed); on one GPU the fused C-ABI call.
    if world > 1:
        from fir_b200.distributed import ShardedOSEM

        sharded = ShardedOSEM(ctx, w.proj, w.vol, prm)
        bp_buf = torch.zeros_like(img)

        def step(s, kk):
            sharded.subiteration(y, img, sens_frames[s], s, kk, bp=bp_buf)
    else:
        def step(s, kk):
            ctx.osem_subiteration(w.proj, y, w.vol, img, sens_frames[s], prm, s, kk)

    # ---- warm-up
    k = 0
    for _ in range(args.warmup):
        step(k % nsub, k + 1)
        k += 1
    torch.cuda.synchronize()
    ctx.synchronize()

    # ---- timed steps
    ctx.set_option(capi.FIR_OPT_TIMING, 1)
    ctx.projector_time(reset=True)
    launches0 = ctx.launch_count
    stream = torch.cuda.current_stream()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    step_counts = []
    kernel_bytes = 0
    gpu_id = str(local)
    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_id) as clocks:
        wall0 = time.perf_counter()
        for i in range(args.steps):
            s = k % nsub
            sb = s_bwd(s)
            step_counts.append(s_fwd[s] + sb)
            # algorithmic bytes of the fused kernel: 4 B per projection step,
            # 8 B per backprojection step, 4 B per LOR of the subset
            kernel_bytes += 4 * s_fwd[s] + 8 * sb + 4 * (nb // nsub)
            flush.zero_()
            starts[i].record(stream)
            step(s, k + 1)
            ends[i].record(stream)
            k += 1
        torch.cuda.synchronize()
        wall = time.perf_counter() - wall0
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.synchronize()
    launches = ctx.launch_count - launches0
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_ms = sum(step_ms)
    kern_ms, kern_n = ctx.projector_time(reset=True)
    ctx.set_option(capi.FIR_OPT_TIMING, 0)
    total_steps = sum(step_counts)
    if dist is not None:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t)
    # every step covers the whole subset, split across the ranks
    value = total_steps / (total_ms / 1000.0)

    hbm, hbm_kind = peaks()
    achieved = (kernel_bytes / kern_n) / (kern_ms / kern_n / 1000.0) / 1e9 if kern_n else None
    prof = profile_traffic()
    traffic = None
    if prof and prof.get("dram_bytes_per_lor"):
        traffic = prof["dram_bytes_per_lor"] * (nb // nsub)
    roofline = {
        "bound": "hbm",
        "kernel": "k_osem_subset (fused projection + ratio + backprojection)",
        "achieved": achieved,
        "peak": hbm,
        "unit": "GB/s",
        "frac": achieved / hbm if achieved else None,
        "peak_kind": f"{hbm_kind} (MEASURED_PEAKS.json hbm_gbs)" if hbm_kind == "measured" else "fallback",
        "traffic": traffic,
        "kernel_ms_per_launch": kern_ms / kern_n if kern_n else None,
        "algorithmic_bytes_per_launch": kernel_bytes / max(1, kern_n),
    }

    result = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32 data, f64 geometry",
        "data": "synthetic (seeded phantom, water attenuation, Poisson counts)",
        "config": bench_config(w, world, nb),
        "osem_s_per_iteration": total_ms / args.steps * nsub / 1000.0,
        "steps_per_subiteration": total_steps / args.steps,
        "wall_s_timed_loop": wall,
        "gpu_launches": launches,
        "roofline": roofline,
        "clocks": {k2: v for k2, v in clocks.summary().items() if k2 != "samples"},
    }

    # ---- the same steps skipping bins with no counts (exact: their ratio is 0),
    # reported beside the headline, which traces every bin as FIR does
    if args.skip_zero_steps > 0:
        ctx.set_option(capi.FIR_OPT_SKIP_ZERO_BINS, 1)
        step(k % nsub, k + 1)  # warm: allocates the list scratch
        k += 1
        sz_steps = 0
        # timed as the headline steps: enqueued back to back, each between its
        # own events after an L2 flush, one synchronisation at the end
        sz_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                     for _ in range(args.skip_zero_steps)]
        torch.cuda.synchronize()
        for a, b in sz_events:
            s = k % nsub
            sz_steps += s_fwd[s] + s_bwd(s)
            flush.zero_()
            a.record(stream)
            step(s, k + 1)
            b.record(stream)
            k += 1
        torch.cuda.synchronize()
        sz_ms = sum(a.elapsed_time(b) for a, b in sz_events)
        ctx.set_option(capi.FIR_OPT_SKIP_ZERO_BINS, 0)
        result["skip_zero_bins"] = {
            "value": sz_steps / (sz_ms / 1000.0),
            "unit": UNIT,
            "ms_per_step": sz_ms / args.skip_zero_steps,
            "steps": args.skip_zero_steps,
            "zero_bin_fraction": float((y == 0).float().mean()),
            "note": "FIR_OPT_SKIP_ZERO_BINS: bins with y = 0 are not traced (their ratio is exactly 0); steps "
                    "counted as for the headline",
        }

    # ---- the same steps with deterministic backprojection (FIR's serial order)
    if args.det_steps > 0:
        det = capi.Context(w.scanner, device=local)
        if w.geometry:
            det.set_option(capi.FIR_OPT_GEOMETRY, w.geometry)
        det.set_option(capi.FIR_OPT_BACKPROJ_MODE, capi.FIR_BACKPROJ_DETERMINISTIC)
        dimg = img.clone()
        det.osem_subiteration(w.proj, y, w.vol, dimg, sens_frames[k % nsub], prm, k % nsub, k + 1)  # warm
        k += 1
        det_steps = 0
        det_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                      for _ in range(args.det_steps)]
        torch.cuda.synchronize()
        for a, b in det_events:
            s = k % nsub
            det_steps += s_fwd[s] + s_bwd(s)
            flush.zero_()
            a.record(stream)
            det.osem_subiteration(w.proj, y, w.vol, dimg, sens_frames[s], prm, s, k + 1)
            b.record(stream)
            k += 1
        torch.cuda.synchronize()
        det_ms = sum(a.elapsed_time(b) for a, b in det_events)
        det.close()
        result["deterministic"] = {
            "value": det_steps / (det_ms / 1000.0),
            "unit": UNIT,
            "ms_per_step": det_ms / args.det_steps,
            "steps": args.det_steps,
            "note": "FIR_BACKPROJ_DETERMINISTIC: contributions sorted per voxel into FIR's serial order "
                    "(bit-identical to single-threaded FIR)",
        }

    # ---- the same steps with the opt-in float traversal (not FIR's arithmetic),
    # and its image error after one iteration against the exact traversal's
    if args.float_steps > 0:
        from fir_b200.geometry import OSEMParams

        fc = capi.Context(w.scanner, device=local)
        if w.geometry:
            fc.set_option(capi.FIR_OPT_GEOMETRY, w.geometry)
        fc.set_option(capi.FIR_OPT_TRAVERSAL, capi.FIR_TRAVERSAL_FLOAT)
        fimg = img.clone()
        fc.osem_subiteration(w.proj, y, w.vol, fimg, sens_frames[k % nsub], prm, k % nsub, k + 1)  # warm
        fc.set_option(capi.FIR_OPT_TIMING, 1)
        fc.projector_time(reset=True)
        f_steps, f_bytes = 0, 0
        f_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                    for _ in range(args.float_steps)]
        torch.cuda.synchronize()
        for a, b in f_events:
            s = k % nsub
            sb = s_bwd(s)
            f_steps += s_fwd[s] + sb
            f_bytes += 4 * s_fwd[s] + 8 * sb + 4 * (nb // nsub)
            flush.zero_()
            a.record(stream)
            fc.osem_subiteration(w.proj, y, w.vol, fimg, sens_frames[s], prm, s, k + 1)
            b.record(stream)
            k += 1
        torch.cuda.synchronize()
        f_ms = sum(a.elapsed_time(b) for a, b in f_events)
        fk_ms, fk_n = fc.projector_time(reset=True)
        fc.set_option(capi.FIR_OPT_TIMING, 0)
        one = OSEMParams(n_iterations=1, n_subsets=nsub, convolution_interval=prm.convolution_interval,
                         fwhm_xyz=list(prm.fwhm_xyz), cut_radius=prm.cut_radius)
        ex = torch.ones(w.vol.shape_zyx, device=dev)
        aux.osem(w.proj, y, w.vol, ex, sens, one)
        fl = torch.ones(w.vol.shape_zyx, device=dev)
        fc.osem(w.proj, y, w.vol, fl, sens, one)
        torch.cuda.synchronize()
        f_err = float((fl.double() - ex.double()).norm() / ex.double().norm())
        fc.close()
        f_achieved = f_bytes / (fk_ms / 1000.0) / 1e9 if fk_ms else None
        result["float_traversal"] = {
            "value": f_steps / (f_ms / 1000.0),
            "unit": UNIT,
            "ms_per_step": f_ms / args.float_steps,
            "kernel_ms_per_launch": fk_ms / fk_n if fk_n else None,
            "roofline_frac": f_achieved / hbm if f_achieved else None,
            "steps": args.float_steps,
            "rel_l2_vs_exact_one_iteration": f_err,
            "note": "FIR_OPT_TRAVERSAL = FIR_TRAVERSAL_FLOAT (opt-in): FIR's double set-up, float loop and "
                    "accumulation; not FIR's arithmetic (voxel lists differ for ~3 % of LORs); steps and "
                    "algorithmic bytes counted as for the headline",
        }

    # ---- end to end through the C ABI with host buffers: one OSEM iteration
    if not args.no_e2e and rank == 0:
        from fir_b200.geometry import OSEMParams

        y_h = torch.empty(nb, dtype=torch.float32, pin_memory=True)
        y_h.copy_(y)
        sens_h = torch.empty(sens.shape, dtype=torch.float32, pin_memory=True)
        sens_h.copy_(sens)
        img_h = torch.empty(w.vol.shape_zyx, dtype=torch.float32, pin_memory=True)
        img_h.copy_(img)
        e2e_steps = 0
        for s in range(nsub):
            e2e_steps += s_fwd[s] + s_bwd(s)
        prm1 = OSEMParams(n_iterations=1, n_subsets=nsub, convolution_interval=prm.convolution_interval,
                          fwhm_xyz=list(prm.fwhm_xyz), cut_radius=prm.cut_radius)
        ctx.osem(w.proj, y_h, w.vol, img_h, sens_h, prm1)  # stage buffers once (warm)
        e2e_s = []
        for _ in range(args.e2e_runs):
            img_h.copy_(img)
            t0 = time.perf_counter()
            ctx.osem(w.proj, y_h, w.vol, img_h, sens_h, prm1)
            e2e_s.append(time.perf_counter() - t0)
        dt = statistics.median(e2e_s)
        h2d = (nb + sens.numel() + nvox) * 4
        result["e2e"] = {
            "value": e2e_steps / dt,
            "unit": UNIT,
            "h2d_bytes_per_step": h2d // nsub,
            "d2h_bytes_per_step": (nvox * 4) // nsub,
            "call": "fir_osem with pinned host buffers, 1 iteration = "
                    f"{nsub} steps, copies inside the timed region; median of {len(e2e_s)} calls",
            "osem_s_per_iteration": dt,
            "osem_s_per_iteration_all": e2e_s,
        }

    if args.batch_runs > 0 and world == 1:
        result["batched"] = batched_section(args, local)
    if args.lbfgs_steps > 0 and world == 1:
        result["autograd"] = autograd_section(args, local)
    if args.large_runs > 0 and world == 1:
        result["large"] = large_section(args, local)

    if not args.no_cpu_baseline and rank == 0 and world == 1:
        try:
            from oracle.bridge import Reference

            ref = Reference()
            ref.threads(os.cpu_count() or 1)
            counts_ref = reference_counts(w, ref, nb)
            r = cpu_reference_run(w, ref, y_host, sens.cpu().numpy(), np.ones(w.vol.shape_zyx, np.float32),
                                  counts_ref, 1)
            result["cpu_baseline"] = {k2: r[k2] for k2 in ("value", "unit", "cores", "kind", "sample")}
            result["cpu_baseline"]["osem_s_per_iteration"] = r["osem_s_per_iteration"]
        except Exception as e:  # noqa: BLE001
            result["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                      "sample": f"unavailable: {e}"}

    if rank == 0:
        print(json.dumps(result))
    ctx.close()
    aux.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
