"""Benchmark of the differentiable forward projection: fwd+bwd rays/s of one
training step (fused projection, MSE loss, hand-written adjoint, Adam update).

Headline workload (the largest configuration that fits one GPU): the thin
slab, a 1024 x 1024 x 256 phantom of 5000 ellipsoids tilted off-axis, 81
tilts on a 1024^2 detector, an adaptive octree refined to depth 6 with about
4096 active leaves, rank-24 VM in BF16 with the decoder 24 -> 64 -> 64 -> 1 on
the tensor cores, 16384-ray batches. The depth-4 / rank-16 workload (256^3
phantom, 61 tilts, 256^2 detector) is measured beside it in the plain FP32
form and the chosen BF16 form, with the seconds to a PSNR target.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). Under torchrun each rank trains on its own ray
batches (ray data parallelism; weak scaling): the BF16 form's gradients are
reduce-scattered, each rank updates its shard of the parameters and the BF16
working copies are all-gathered (dp.ShardedAdam); the plain FP32 form
all-reduces its gradients. `--impl reference` times the CPU restatement of
the reference path (the reference itself has no CPU path and cannot be built
here) on all host cores, on the headline workload.
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd rays/s"
# samples per ray of the learned proposal on the depth-4 workload: the
# smallest budget whose projection error against the uniform judge stays
# within the 1% gate on its tilt series (0.9-1.0% at 160, 1.0-1.4% at 128)
PROPOSAL_BUDGET = 160


def workload_name(cfg):
    if cfg.name == "C5":
        return ("C5: 1024x1024x256 slab phantom (5000 ellipsoids, off-axis tilt "
                f"{cfg.off_axis_deg:.2f} deg), 81 tilts x 1024^2 detector, adaptive octree to depth 6 "
                f"(~{cfg.target_leaves} leaves), rank-24 VM 17^2 planes, decoder 24->64->64->1 BF16, "
                f"{cfg.rays_per_batch}-ray batch, {cfg.max_samples_per_node} samples/leaf-diagonal")
    return ("C2: 256^3 phantom (200 ellipsoids), 61 tilts x 256^2 detector, octree depth 4 (4096 leaves), "
            "rank-16 VM 17^2 planes, decoder 16->64->64->1, 16384-ray batch, "
            f"{cfg.max_samples_per_node} samples/leaf-diagonal")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rays", type=int, default=16384)
    ap.add_argument("--cpu-rays", type=int, default=128, help="rays per CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-psnr", action="store_true", help="skip the seconds-to-PSNR runs")
    ap.add_argument("--no-psnr30", action="store_true", help="skip the seconds-to-30 dB runs")
    ap.add_argument("--no-gate", action="store_true", help="skip the proposal's 400-step gate run on C5")
    ap.add_argument("--psnr-target", type=float, default=18.0)
    ap.add_argument("--psnr-epochs", type=int, default=3)
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="only run this many forward + backward projections of the workload's BF16 form (no "
                         "timing, no JSON line): the program a profiler captures")
    ap.add_argument("--workload", default="C5", help="configuration of --profile-steps (C2 or C5)")
    return ap.parse_args()


# ----------------------------------------------------------------------------
# workload
# ----------------------------------------------------------------------------
def workload_config(name="C5"):
    from adaptivetensordf_b200.synthetic import CONFIGS

    return CONFIGS[name]


def make_batches(cfg, R, nb, seed, device=None):
    """nb batches of R rays of the configuration's tilt series (random tilt
    and pixel) with the phantom's analytic line integrals as targets
    (computed on `device` when one is given)."""
    from adaptivetensordf_b200 import synthetic as syn

    ph = syn.config_phantom(cfg, 1001)
    out = []
    for b in range(nb):
        o, d = syn.random_ray_batch(cfg, R, seed + b)
        y = syn.analytic_projection(ph, o, d, device=device).astype(np.float32)
        out.append((o, d, y))
    return out


# ----------------------------------------------------------------------------
# clocks
# ----------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up (driver and NVML initialisation, slow on a
            # fresh machine) must not overlap the timed region: wait for its
            # first sample before returning
            t0 = time.time()
            while not self.lines and self.proc.poll() is None and time.time() - t0 < 20.0:
                time.sleep(0.05)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
# CPU baseline (the oracle port of the reference path)
# ----------------------------------------------------------------------------
def oracle_tree(cfg):
    """The workload's tree in the oracle's form: every depth-tree_depth node
    active, or the adaptive leaves of the configuration's phantom."""
    from adaptivetensordf_b200 import synthetic as syn
    from oracle import oracle as O

    t = O.tree_build(cfg.tree_depth)
    if cfg.target_leaves:
        leaves, _ = syn.adaptive_leaves(cfg, syn.config_phantom(cfg, 1001), t["node_position_min"],
                                        t["node_position_max"], t["node_children"], t["node_depth"])
        act = np.zeros(len(t["node_depth"]), np.int32)
        act[leaves] = 1
        O.set_active(t, act)
    else:
        O.set_active_depth(t, cfg.tree_depth)
    return t


def batch_counts(cfg, t, R):
    """Segments and uniform samples of the workload's first batch (the
    config keys both arms report)."""
    from oracle import oracle as O

    from adaptivetensordf_b200 import synthetic as syn

    o, d = syn.random_ray_batch(cfg, R, 1004)
    segs = O.ray_segments(t, o, d, cfg.max_samples_per_node)
    return len(segs["n"]), int(segs["n"].sum())


def cpu_baseline(cfg, t, R, steps=1, seed=77):
    """The oracle's plain FP32 training step (segments, samples, VM field,
    decoder, integral, MSE loss, hand-written adjoint) on R rays of the
    workload, all OpenMP threads."""
    from oracle import oracle as O

    N = len(t["active_node_ids"])
    rng = np.random.default_rng(1003)
    C, G = cfg.channels, cfg.grid
    lines = cfg.lines()
    field = {"planes": [rng.uniform(-0.5, 0.5, (N, C, G, G)).astype(np.float32) for _ in range(3)],
             "lines": [rng.uniform(-0.5, 0.5, (1, C, L, 1)).astype(np.float32) for L in lines],
             "leaf_slot": t["node_active_prefix_sum"]}
    dims = [C] + cfg.hidden + [1]
    mlp = {"layers": [(rng.normal(0, math.sqrt(2 / dims[i]), (dims[i + 1], dims[i])).astype(np.float32),
                       rng.uniform(-1, 1, dims[i + 1]).astype(np.float32) / math.sqrt(dims[i]))
                      for i in range(len(dims) - 1)], "act": "silu", "last_act": "softplus", "beta": 2.0}
    batches = make_batches(cfg, R, steps, seed)
    times = []
    for o, d, y in batches:
        t0 = time.perf_counter()
        O.train_step(t, field, mlp, o, d, y, cfg.max_samples_per_node, 1234)
        times.append(time.perf_counter() - t0)
    return {"value": R / statistics.median(times), "unit": "rays/s", "cores": O.num_threads(), "kind": "port",
            "sample": f"{R} rays of the {cfg.name} workload per step (same tree, field shapes, decoder, samples "
                      f"per leaf diagonal), FP32, median of {len(times)} steps, {O.num_threads()} OpenMP threads"}


def shared_config(cfg, leaves, nseg, nsamp):
    """Config keys both arms report for the same workload."""
    return {"workload": workload_name(cfg), "rays_per_gpu_step": cfg.rays_per_batch, "samples_per_step": nsamp,
            "segments_per_step": nseg, "leaves": leaves,
            "l2": "inputs larger than L2 (BF16 factors read and FP32 gradients written per step)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    cfg = workload_config()
    t = oracle_tree(cfg)
    nseg, nsamp = batch_counts(cfg, t, cfg.rays_per_batch)
    R = args.cpu_rays
    for _ in range(max(args.warmup, 0) and 1):
        cpu_baseline(cfg, t, R, 1, seed=5)
    t0 = time.perf_counter()
    cb = cpu_baseline(cfg, t, R, max(args.steps, 1), seed=9)
    wall = time.perf_counter() - t0
    line = {"metric": METRIC, "value": cb["value"], "unit": "rays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * R / cb["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": shared_config(cfg, len(t["active_node_ids"]), nseg, nsamp),
            "parallelism": f"CPU, {cb['cores']} OpenMP threads", "cpu_rays_per_step": R, "impl": "reference",
            "cpu_baseline": {k: cb[k] for k in ("kind", "cores", "sample", "value", "unit")},
            "e2e": {"value": cb["value"], "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------
def measure_proposal(args, tree, cfg, dev_batches, nb, stream, budget):
    """Steady-state step of the BF16 form through the learned proposal's
    samples (budget per ray; segments, proposal MLP, allocation and sampling
    included), and the cost of one judge step (uniform binned pass +
    proposal training), which the schedule runs every 10 steps while the
    proposal is in use."""
    import torch

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn
    from adaptivetensordf_b200.optim import Adam

    geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=1003)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    params = syn.parameters(geo)
    opt = Adam(params, lr=1e-3, geometry=geo)  # also writes the BF16 working copies
    ps = ab.ProposalSampler(tree.NumNodes(), 64, 3, 1005, "cuda")
    ps.budget = budget
    ps.precision = "bf16"  # the proposal MLP on the tensor cores, as in the BF16 form's schedule
    padam = torch.optim.Adam(ps.parameters(), lr=3e-3)

    def step(k, judge):
        o, d, y = dev_batches[k % nb]
        rays = ab.RayList(o, d)
        if judge:
            img = ps.ProjectUniformBinned(tree, geo, rays, cfg.max_samples_per_node, 1 + k)
        else:
            img = ps.Project(tree, geo, rays, 1 + k)
        loss, gimg = ab.MseLossAndGrad(img, y, 1.0)
        img.backward(gimg)
        opt.step()
        opt.zero_grad(set_to_none=True)
        if judge:
            padam.zero_grad()
            ps.ComputeGradients(tree)
            padam.step()

    for k in range(max(args.warmup, 3)):
        step(k, k == 0)
    res = {}
    for name, judge in (("proposal_step", False), ("judge_step", True)):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(args.steps):
            step(100 + k, judge)
        e1.record(stream)
        torch.cuda.synchronize()
        res[name + "_ms"] = e0.elapsed_time(e1) / args.steps
    geo.CheckErrors()
    R = dev_batches[0][0].shape[0]
    amort = (9 * res["proposal_step_ms"] + res["judge_step_ms"]) / 10
    res.update({"budget_per_ray": budget,
                "rays_per_s_proposal_steps": R / (res["proposal_step_ms"] * 1e-3),
                "rays_per_s_with_judge_every_10": R / (amort * 1e-3)})
    del geo, opt, params, ps
    return res


def proposal_gate(tree, cfg, dev_batches, budget, steps=400):
    """Does the proposal hold the 1% gate at this budget? Trains the BF16
    form from the seeded initialisation through the proposal schedule (judge
    every 10th step, every step in the 20-step warm-up) for `steps` steps on
    the workload's batches and reports the schedule's counters, the last
    judge's projection error and the error every 100 steps."""
    import torch

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn
    from adaptivetensordf_b200.optim import Adam
    from adaptivetensordf_b200.proposal import ProposalSchedule

    geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=1003, init_scale=0.05)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    opt = Adam([{"params": list(geo.planes) + list(geo.lines), "lr": 0.01},
                {"params": list(geo.decoder_weight) + list(geo.decoder_bias), "lr": 5e-4}], geometry=geo)
    prop = ProposalSchedule(tree, geo, cfg.max_samples_per_node, budget=budget)
    trace = []
    t0 = time.perf_counter()
    for k in range(steps):
        o, d, y = dev_batches[k % len(dev_batches)]
        img = prop.project(ab.RayList(o, d), 1 + k, y)
        loss, gimg = ab.MseLossAndGrad(img, y, 1.0)
        img.backward(gimg)
        opt.step()
        opt.zero_grad(set_to_none=True)
        if k % 100 == 99:
            trace.append([k + 1, prop.last_error])
    torch.cuda.synchronize()
    geo.CheckErrors()
    res = {"budget_per_ray": budget, "steps": steps, "gate": prop.gate, "error_trace": trace,
           "wall_s": time.perf_counter() - t0, **prop.stats()}
    del geo, opt, prop
    return res


def projection_psnr_race(tree, cfg, target_db=49.0, steps=3000, nb=48, budget=64, every=100):
    """Wall time of the BF16 form to a held-out projection PSNR on the
    workload, with the uniform sampler and through the learned proposal
    (`budget` samples per ray, judge every 10th step): both train from the
    same seeded initialisation on the same `nb` batches; every `every` steps
    the uniform projection of a held-out batch of 16384 rays is compared
    with its analytic targets (10 log10(peak^2 / MSE), peak = the batch's
    largest target), outside the clock. The projection domain stands in for
    the volume PSNR here: voxelising the 1024 x 1024 x 256 slab of 5000
    ellipsoids for a volume reference would cost more than the whole run."""
    import torch

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn
    from adaptivetensordf_b200.optim import Adam
    from adaptivetensordf_b200.proposal import ProposalSchedule

    R = cfg.rays_per_batch
    batches = [tuple(torch.from_numpy(a).cuda() for a in b) for b in make_batches(cfg, R, nb, 7000, device="cuda")]
    vo, vd, vy = (torch.from_numpy(a).cuda() for a in make_batches(cfg, R, 1, 9999, device="cuda")[0])
    peak = float(vy.max())
    M = cfg.max_samples_per_node

    def run(with_prop):
        geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=1003, init_scale=0.05)
        geo.precision = "bf16"
        geo.RefreshLowPrecision()
        opt = Adam([{"params": list(geo.planes) + list(geo.lines), "lr": 0.01},
                    {"params": list(geo.decoder_weight) + list(geo.decoder_bias), "lr": 5e-4}], geometry=geo)
        prop = ProposalSchedule(tree, geo, M, budget=budget) if with_prop else None
        clock, reached, best, curve = 0.0, None, -1.0, []
        torch.cuda.synchronize()
        for k in range(steps):
            t1 = time.perf_counter()
            o, d, y = batches[k % nb]
            rays = ab.RayList(o, d)
            img = prop.project(rays, 1 + k, y) if prop else geo.ProjectRays(tree, rays, M, 1 + k)
            loss, gimg = ab.MseLossAndGrad(img, y, 1.0)
            img.backward(gimg)
            opt.step()
            opt.zero_grad(set_to_none=True)
            if (k + 1) % every:
                clock += time.perf_counter() - t1
                continue
            torch.cuda.synchronize()
            clock += time.perf_counter() - t1
            with torch.no_grad():
                v = geo.ProjectRays(tree, ab.RayList(vo, vd), M, 0).reshape(-1)
                db = 10.0 * math.log10(peak * peak / float(((v - vy) ** 2).mean()))
            best = max(best, db)
            curve.append([k + 1, round(clock, 3), round(db, 3)])
            if db >= target_db:
                reached = clock
                break
        geo.CheckErrors()
        out = {"seconds": reached, "steps": curve[-1][0], "best_db": best, "curve": curve[::5]}
        if prop:
            out.update({k: v for k, v in prop.stats().items() if k in ("judge_steps", "proposal_steps",
                                                                         "uniform_steps", "proposal_error")})
        return out

    res = {"target_db": target_db, "metric": "held-out projection PSNR (16384 rays, analytic targets)",
           "workload": cfg.name, "budget_per_ray": budget, "bf16": run(False), "bf16+prop": run(True)}
    if res["bf16"]["seconds"] and res["bf16+prop"]["seconds"]:
        res["ratio_bf16_over_bf16+prop"] = res["bf16"]["seconds"] / res["bf16+prop"]["seconds"]
    del batches
    torch.cuda.empty_cache()
    return res


def time_entry_points(tree, geo, o, d, M, seed, reps=10):
    """GPU time of the fused forward and backward entry points alone, called
    through the C ABI with preallocated gradients and the forward's
    workspace (the same segments as a training step), CUDA events on the
    launching stream. The backward call is the tensor-core backward kernel
    plus a few memsets; the forward call includes the ray/leaf segment pass
    and the bucketing before its kernel."""
    import ctypes as ct

    import torch

    from adaptivetensordf_b200 import capi

    L = capi.lib()
    st = torch.cuda.current_stream()
    sp = ct.c_void_p(st.cuda_stream)
    t = capi.tree_struct(tree)
    f, keep_f = capi.field_struct_bf16(geo) if geo.precision == "bf16" else capi.field_struct(geo)
    m, keep_m = capi.mlp_struct(geo)
    fg, mg, keep_g = capi.grad_structs(geo)
    R = o.shape[0]
    size = ct.c_size_t(0)
    assert L.atdf_project_workspace_size(R, t.max_depth, t.ns, f.num_slots, 1, ct.byref(size)) == 0
    ws = torch.empty(size.value, dtype=torch.uint8, device="cuda")
    img = torch.empty(1, R, device="cuda")
    gimg = torch.full((1, R), 1.0 / R, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")

    def fwd():
        assert L.atdf_project_forward(ct.byref(t), ct.byref(f), ct.byref(m), capi.ptr(o), capi.ptr(d), R, M, seed,
                                      capi.ptr(img), capi.ptr(ws), size.value, capi.ptr(err), sp) == 0

    def bwd():
        assert L.atdf_project_backward(ct.byref(t), ct.byref(f), ct.byref(m), capi.ptr(o), capi.ptr(d), R, M, seed,
                                       capi.ptr(gimg), ct.byref(fg), ct.byref(mg), capi.ptr(ws), size.value,
                                       capi.ptr(err), sp) == 0

    out = {}
    for name, fn in (("forward", fwd), ("backward", bwd)):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    assert err.item() == 0, err.item()
    del keep_f, keep_m, keep_g
    return out


def device_copy_gbs(stream, nbytes=1 << 30, reps=10):
    """This GPU's device-to-device copy bandwidth (read + write bytes per
    second, 1 GiB buffers, CUDA events), reported beside the roofline's peak
    for context."""
    import torch

    a = torch.empty(nbytes // 4, dtype=torch.float32, device="cuda").fill_(1.0)
    b = torch.empty_like(a)
    for _ in range(3):
        b.copy_(a)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        b.copy_(a)
    e1.record(stream)
    torch.cuda.synchronize()
    gbs = 2 * nbytes * reps / (e0.elapsed_time(e1) * 1e-3) / 1e9
    del a, b
    torch.cuda.empty_cache()
    return gbs


def time_to_psnr(args):
    """Training wall time (evaluations excluded) until the voxel-grid PSNR
    reaches the target, for the plain FP32 and the BF16 forms, on the C2
    tilt series (seeded synthetic phantom, FP64 Siddon projections, noise)."""
    from adaptivetensordf_b200 import recon
    from adaptivetensordf_b200.synthetic import CONFIGS

    cfg = CONFIGS["C2"]
    data = recon.make_tilt_series(cfg)
    out = {"target_db": args.psnr_target, "config": "C2 tilt series, 16384-ray batches, eval every 61 steps"}
    for form in ("fp32", "bf16", "bf16+prop"):
        opt = recon.TrainOptions(epochs=args.psnr_epochs, batch=cfg.rays_per_batch,
                                 max_samples_per_node=cfg.max_samples_per_node, eval_every=61,
                                 target_psnr=args.psnr_target, init_scale=0.05, budget=PROPOSAL_BUDGET)
        recs, reached = recon.train(cfg, form, data, opt)
        out[form] = {"seconds": reached, "best_psnr": max(r["psnr"] for r in recs), "steps": recs[-1]["step"]}
        if form.endswith("+prop"):
            out[form].update({k: recs[-1][k] for k in ("judge_steps", "proposal_steps", "uniform_steps",
                                                        "proposal_error")})
    for form in ("bf16", "bf16+prop"):
        if out["fp32"]["seconds"] and out[form]["seconds"]:
            out[f"ratio_fp32_over_{form}"] = out["fp32"]["seconds"] / out[form]["seconds"]
    # the adaptive recipe of the configuration: a depth-3 start refined toward
    # depth 4 (greedy structure optimisation, budget 1024 leaves, every 2 epochs)
    ad = {"target_db": args.psnr_target + 0.6,
          "recipe": "start at depth 3 (512 leaves), refine every 2 epochs, budget 1024 leaves"}
    for form in ("fp32", "bf16"):
        opt = recon.TrainOptions(epochs=args.psnr_epochs + 1, batch=cfg.rays_per_batch,
                                 max_samples_per_node=cfg.max_samples_per_node, eval_every=61,
                                 target_psnr=ad["target_db"], init_scale=0.05, start_depth=3, refine_every=2,
                                 max_active_nodes=1024)
        recs, reached = recon.train(cfg, form, data, opt)
        ad[form] = {"seconds": reached, "best_psnr": max(r["psnr"] for r in recs), "steps": recs[-1]["step"]}
    if ad["fp32"]["seconds"] and ad["bf16"]["seconds"]:
        ad["ratio_fp32_over_bf16"] = ad["fp32"]["seconds"] / ad["bf16"]["seconds"]
    out["adaptive_tree"] = ad
    del data
    return out


# the 30 dB workload: the C2 phantom and model on a full-angle, noise-free
# series (90 tilts at 2 deg, +-89 deg), learning-rate decay 0.99 per epoch,
# PSNR evaluated every 360 steps, at most 420 s of training per form
PSNR30 = {"angles": 90, "angle_step": 2.0, "noise": 0.0, "jitter": 0.0, "lr_decay": 0.99, "epochs": 60,
          "eval_every": 360, "time_limit": 420.0, "proposal_budget": 128, "residual_gate": 0.5}


def time_to_psnr30():
    """Seconds to 30 dB of the plain FP32 form, the BF16 form and the BF16
    form with the learned proposal, on the 30 dB workload (PSNR30)."""
    from adaptivetensordf_b200 import recon
    from adaptivetensordf_b200.synthetic import CONFIGS

    w = PSNR30
    cfg = dataclasses.replace(CONFIGS["C2"], angles=w["angles"], angle_step=w["angle_step"], noise=w["noise"],
                              jitter=w["jitter"])
    data = recon.make_tilt_series(cfg)
    out = {"target_db": 30.0, "workload": "C2 phantom and model, 90 noise-free tilts at 2 deg (+-89 deg), "
           "16384-ray batches, lr decay 0.99 per epoch, PSNR every 360 steps", **w}
    for form in ("fp32", "bf16", "bf16+prop"):
        opt = recon.TrainOptions(epochs=w["epochs"], batch=cfg.rays_per_batch,
                                 max_samples_per_node=cfg.max_samples_per_node, eval_every=w["eval_every"],
                                 target_psnr=30.0, init_scale=0.05, lr_decay=w["lr_decay"],
                                 time_limit=w["time_limit"], budget=w["proposal_budget"],
                                 residual_gate=w["residual_gate"])
        recs, reached = recon.train(cfg, form, data, opt)
        out[form] = {"seconds": reached, "best_psnr": max(r["psnr"] for r in recs), "steps": recs[-1]["step"],
                     "train_seconds": recs[-1]["t"]}
        if form.endswith("+prop"):
            out[form].update({k: recs[-1][k] for k in ("judge_steps", "proposal_steps", "uniform_steps",
                                                        "proposal_error")})
    for form in ("bf16", "bf16+prop"):
        if out["fp32"]["seconds"] and out[form]["seconds"]:
            out[f"ratio_fp32_over_{form}"] = out["fp32"]["seconds"] / out[form]["seconds"]
    del data
    return out


def step_bytes(cfg, n_slots, nseg, R):
    """Algorithmic bytes of the BF16 backward launch: the BF16 planes read,
    the FP32 plane gradient written, the segment records and the rays."""
    F = 3 * cfg.channels * cfg.grid * cfg.grid  # plane elements per leaf
    return n_slots * F * 2 + n_slots * F * 4 + nseg * 24 + R * 32


def measure_form(args, tree, cfg, form, dev_batches, host_batches, world, sampler=None):
    """One form's training step on a workload: device-timed K steps
    (inputs resident), the same through the public API with pinned host
    inputs and the loss read back (e2e), the forward / backward autograd calls
    and the fused entry points timed alone."""
    import torch

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import dp
    from adaptivetensordf_b200 import synthetic as syn
    from adaptivetensordf_b200.optim import Adam

    import torch.distributed as dist

    stream = torch.cuda.current_stream()
    nb = len(dev_batches)
    M = cfg.max_samples_per_node
    geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=1003)
    bf16 = form == "bf16"
    if bf16:
        geo.precision = "bf16"
        geo.RefreshLowPrecision()
    params = syn.parameters(geo)
    # the BF16 form's Adam also writes the BF16 working copies, on a side
    # stream so that the next step's segment pass overlaps it; the plain
    # FP32 form keeps torch's fused Adam
    sharded = bf16 and world > 1
    if sharded:
        # ray data parallelism with the sharded step: reduce-scatter of the
        # gradients, Adam on this rank's shard, all-gather of the BF16 copies
        twins = list(geo.planes_bf16) + list(geo.lines_bf16)
        opt = dp.ShardedAdam(params, world, int(os.environ.get("RANK", "0")), lr=1e-3,
                             working={i: twins[i] for i in range(6)})
        join = lambda: None  # noqa: E731
    else:
        opt = Adam(params, lr=1e-3, geometry=geo, stream=torch.cuda.Stream()) if bf16 else \
            torch.optim.Adam(params, lr=1e-3, fused=True)
        join = opt.wait if bf16 else (lambda: None)  # the timed region ends after the last update

    def step(o, d, y, k):
        rays = ab.RayList(o, d)
        img = geo.ProjectRays(tree, rays, M, 1 + k)
        loss, gimg = ab.MseLossAndGrad(img, y, 1.0)
        img.backward(gimg)
        if sharded:
            opt.step()
            for p in params:
                p.grad = None
        else:
            dp.allreduce_gradients(params, world)
            opt.step()
            opt.zero_grad(set_to_none=True)
        return loss

    for k in range(args.warmup):
        step(*dev_batches[k % nb], k)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.steps):
        step(*dev_batches[k % nb], 100 + k)
    join()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        dist.barrier()
    # end to end through the public API with host buffers: H2D of the
    # batch, D2H of the loss, every step
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    loss_host = torch.zeros(1, dtype=torch.float64).pin_memory()

    def e2e_step(k, base):
        o, d, y = host_batches[k % nb]
        og, dg, yg = o.cuda(non_blocking=True), d.cuda(non_blocking=True), y.cuda(non_blocking=True)
        loss = step(og, dg, yg, base + k)
        loss_host.copy_(loss.reshape(1), non_blocking=True)

    for k in range(args.warmup):  # the copies' first use of the pinned buffers is not timed
        e2e_step(k, 300)
    torch.cuda.synchronize()
    h0.record(stream)
    for k in range(args.steps):
        e2e_step(k, 200)
    join()
    h1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = h0.elapsed_time(h1) / args.steps
    clocks = sampler.stop() if sampler else None
    # forward and backward autograd calls timed alone (CUDA events on the
    # launching stream); two more forward passes (no autograd) are queued
    # between a forward and its backward so the GPU still has work while the
    # host runs the autograd engine's part of the backward call
    reps = 5
    o, d, y = dev_batches[0]
    rays = ab.RayList(o, d)
    evs = []
    for k in range(reps + 1):  # the first repetition warms the allocator up
        f0, f1, b0, b1 = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        opt.zero_grad(set_to_none=True)
        f0.record(stream)
        img = geo.ProjectRays(tree, rays, M, 7)
        f1.record(stream)
        gimg = torch.ones_like(img)
        with torch.no_grad():
            for _ in range(2):
                geo.ProjectRays(tree, rays, M, 7)
        b0.record(stream)
        img.backward(gimg)
        b1.record(stream)
        evs.append((f0, f1, b0, b1))
    torch.cuda.synchronize()
    tf = sum(f0.elapsed_time(f1) for f0, f1, _, _ in evs[1:]) / reps
    tb = sum(b0.elapsed_time(b1) for _, _, b0, b1 in evs[1:]) / reps
    entry = time_entry_points(tree, geo, o, d, M, 7)
    geo.CheckErrors()
    del geo, opt, params
    torch.cuda.empty_cache()
    return {"ms": ms, "ms_e2e": ms_e2e, "forward_call_ms": tf, "backward_call_ms": tb,
            "forward_entry_ms": entry["forward"], "backward_entry_ms": entry["backward"], "clocks": clocks}


def prepare_workload(cfg, R, rank, nb=4):
    import torch

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn

    if cfg.target_leaves:
        tree = syn.adaptive_tree(cfg, syn.config_phantom(cfg, 1001), device="cuda")
    else:
        tree = syn.make_tree(cfg.tree_depth, device="cuda")
    batches = make_batches(cfg, R, nb, 1004 + 1000 * rank, device="cuda")
    # device-resident inputs (value) and pinned host inputs (e2e)
    dev = [(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda(), torch.from_numpy(y).cuda()[None])
           for o, d, y in batches]
    host = [(torch.from_numpy(o).pin_memory(), torch.from_numpy(d).pin_memory(),
             torch.from_numpy(y)[None].pin_memory()) for o, d, y in batches]
    sg = tree.RaySegments(ab.RayList(*dev[0][:2]), cfg.max_samples_per_node)
    return tree, dev, host, int(sg.num_segments), int(sg.num_samples)


def run_ours(args, rank, world):
    import torch
    import torch.distributed as dist

    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    stream = torch.cuda.current_stream()
    R = args.rays
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    tpeak = peaks.get("bf16_tflops_sustained", 1400.0)

    # headline: the C5 slab in the chosen BF16 form
    cfg = dataclasses.replace(workload_config("C5"), rays_per_batch=R)
    tree, dev, host, nseg, nsamp = prepare_workload(cfg, R, rank)
    n_slots = int(tree.NumActiveNodes())
    sampler = ClockSampler(local)
    r5 = measure_form(args, tree, cfg, "bf16", dev, host, world, sampler)
    prop5 = measure_proposal(args, tree, cfg, dev, len(dev), stream, 64) if world == 1 else None
    if prop5 is not None and not args.no_gate:
        prop5["gate_run"] = proposal_gate(tree, cfg, dev, 64)
    race5 = projection_psnr_race(tree, cfg) if (world == 1 and not args.no_psnr) else None
    del tree, dev, host

    # the depth-4 / rank-16 workload: plain FP32 against the chosen form
    cfg2 = dataclasses.replace(workload_config("C2"), rays_per_batch=R)
    tree2, dev2, host2, nseg2, nsamp2 = prepare_workload(cfg2, R, rank)
    n_slots2 = int(tree2.NumActiveNodes())
    r2 = measure_form(args, tree2, cfg2, "bf16", dev2, host2, world)
    r2_32 = measure_form(args, tree2, cfg2, "fp32", dev2, host2, world)
    prop2 = measure_proposal(args, tree2, cfg2, dev2, len(dev2), stream, PROPOSAL_BUDGET) if world == 1 else None
    del tree2, dev2, host2
    copy_gbs = device_copy_gbs(stream) if world == 1 else None
    psnr = time_to_psnr(args) if (world == 1 and not args.no_psnr) else None
    psnr30 = time_to_psnr30() if (world == 1 and not args.no_psnr and not args.no_psnr30) else None

    vals = torch.tensor([r5["ms"], r5["ms_e2e"], r2["ms"], r2_32["ms"]], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(vals, op=dist.ReduceOp.MAX)
    ms, ms_e2e, ms2, ms2_32 = vals.tolist()
    if rank != 0:
        return

    def rooflines(cfg_, slots, nseg_, nsamp_, r):
        """The dominant kernel (the BF16 backward, its entry point timed
        alone) against the HBM and the tensor-core peaks."""
        kms = r["backward_entry_ms"]
        assert kms <= r["ms"], (kms, r["ms"])  # a kernel of the step cannot outlast the step
        nbytes = step_bytes(cfg_, slots, nseg_, R)
        achieved = nbytes / (kms * 1e-3) / 1e9
        dims = [cfg_.channels] + list(cfg_.hidden) + [1]
        flop_fwd = 2 * sum(a * b for a, b in zip(dims[:-1], dims[1:]))  # decoder FLOP per sample, forward
        flop = 3 * flop_fwd * nsamp_  # recomputed forward + backward (two GEMMs per layer)
        tfl = flop / (kms * 1e-3) / 1e12
        hbm_line = {"bound": "hbm", "kernel": "fused backward (tcgen05), atdf_project_backward timed alone",
                    "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                    "algorithmic_bytes": nbytes, "kernel_ms": kms,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                    else "fallback 6650 GB/s"}
        tensor_line = {"bound": "tensor", "kernel": "fused backward (tcgen05 decoder GEMMs)", "achieved": tfl,
                       "peak": tpeak, "unit": "TFLOP/s", "frac": tfl / tpeak, "flop_per_launch": flop,
                       "flop_per_sample": 3 * flop_fwd,
                       "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)"
                       if "bf16_tflops_sustained" in peaks else "fallback 1400 TFLOP/s (sustained)"}
        return hbm_line, tensor_line

    roof5, troof5 = rooflines(cfg, n_slots, nseg, nsamp, r5)
    roof2, troof2 = rooflines(cfg2, n_slots2, nseg2, nsamp2, r2)
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one
    # tcgen05 backward launch on the depth-4 workload at 16384 rays, from a
    # single-pass ncu capture (its summary is named in traffic_source); the
    # gradient writes still in L2 when the kernel ends are not counted there
    roof2["traffic"] = 129719040 + 179244288 if R == 16384 else None
    roof2["traffic_source"] = "profiles/tc_backward_dram_c2_16384rays.md" if R == 16384 else None
    # the same for the C5 rank-24 backward (full-size capture, 3 launches)
    roof5["traffic"] = 177041835 + 283314176 if R == 16384 else None
    roof5["traffic_source"] = "profiles/launches_c5_bf16_16384rays.md" if R == 16384 else None
    # this library's kernels per uniform training step of the BF16 form: 12
    # for sampling, bucketing (slot order, item queue) and the forward, the
    # loss, 2 for the backward and one Adam launch for the 12 parameters
    launches_per_step = 16
    h2d = sum(t.numel() * t.element_size() for t in make_host_shapes(R))
    line = {
        "metric": METRIC,
        "value": world * R / (ms * 1e-3),
        "unit": "rays/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16",
        "data": "synthetic",
        "config": shared_config(cfg, n_slots, nseg, nsamp),
        "parallelism": f"ray data parallel x{world}" if world > 1 else "single GPU",
        "form": "chosen: BF16 factors, tcgen05 decoder GEMMs (FP32 accumulation), hand-written adjoint, fused "
                "leaf-major; Adam on FP32 masters",
        "e2e": {"value": world * R / (ms_e2e * 1e-3), "unit": "rays/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 8},
        "roofline": {**roof5, "copy_gbs_this_gpu": copy_gbs},
        "roofline_tensor": troof5,
        "kernels_ms": {k: r5[k] for k in ("forward_call_ms", "backward_call_ms", "forward_entry_ms",
                                          "backward_entry_ms")},
        "samples_per_s": world * nsamp / (ms * 1e-3),
        "gpu_launches": launches_per_step * args.steps,
        "clocks": r5["clocks"],
        "c2": {"workload": workload_name(cfg2), "leaves": n_slots2, "samples_per_step": nsamp2,
               "segments_per_step": nseg2,
               "bf16": {"value": world * R / (ms2 * 1e-3), "ms_per_step": ms2,
                        "e2e_value": world * R / (r2["ms_e2e"] * 1e-3),
                        "kernels_ms": {k: r2[k] for k in ("forward_call_ms", "backward_call_ms",
                                                          "forward_entry_ms", "backward_entry_ms")},
                        "roofline": roof2, "roofline_tensor": troof2},
               "plain_fp32": {"value": world * R / (ms2_32 * 1e-3), "ms_per_step": ms2_32,
                              "e2e_value": world * R / (r2_32["ms_e2e"] * 1e-3),
                              "kernels_ms": {k: r2_32[k] for k in ("forward_call_ms", "backward_call_ms",
                                                                   "forward_entry_ms", "backward_entry_ms")}},
               "speedup_bf16_vs_plain_fp32": ms2_32 / ms2},
    }
    if prop5:
        line["proposal_form"] = prop5
    if prop2:
        line["c2"]["proposal_form"] = {**prop2, "note": "the proposal is used only while its projection error "
                                       "against the uniform judge is <= 1%"}
    if psnr:
        line["seconds_to_psnr"] = psnr
    if psnr30:
        line["seconds_to_30db"] = psnr30
    if race5:
        line["proposal_form"]["seconds_to_projection_psnr"] = race5
    if not args.no_cpu_baseline and world == 1:  # the CPU baseline and the checker run at N = 1 only
        t = oracle_tree(cfg)
        line["cpu_baseline"] = cpu_baseline(cfg, t, args.cpu_rays, 3)
        # the FP64 oracle as the checker of the BF16 form's error (C3 asks
        # for it; the C5 shapes beside it)
        line["bf16_err_vs_fp64"] = {"C3": bf16_error_vs_oracle(workload_config("C3")),
                                    "C5": bf16_error_vs_oracle(cfg)}
    print(json.dumps(line), flush=True)


def bf16_error_vs_oracle(cfg, R=256, seed=4321):
    """Relative L2 error of the BF16 form's projection and gradients (the
    tensor-core kernels) against the FP64 oracle on the same samples of R
    rays of the workload: `vs_bf16_params` with the oracle on the
    BF16-rounded factors and weights (the decoder's BF16 arithmetic alone),
    `vs_fp32_params` with the FP32 parameters (what the precision form costs
    in total)."""
    import torch

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn
    from oracle import oracle as O

    if cfg.target_leaves:
        tree = syn.adaptive_tree(cfg, syn.config_phantom(cfg, 1001), device="cuda")
    else:
        tree = syn.make_tree(cfg.tree_depth, device="cuda")
    geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=1003)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    o, d = syn.random_ray_batch(cfg, R, seed)
    M = cfg.max_samples_per_node
    img = geo.ProjectRays(tree, ab.RayList(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda()), M, seed)
    gi = np.random.default_rng(seed).normal(size=(1, R))
    img.backward(torch.from_numpy(gi.astype(np.float32)).cuda())
    geo.CheckErrors()
    td, fd, md = syn.tree_dict(tree), syn.field_dict(geo, tree), syn.mlp_dict(geo)

    def bf(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(torch.bfloat16).to(torch.float64).numpy()

    fd_b = {**fd, "planes": [bf(p) for p in fd["planes"]], "lines": [bf(x) for x in fd["lines"]]}
    md_b = {**md, "layers": [(bf(w), b.astype(np.float64)) for w, b in md["layers"]]}
    md_b["layers"][-1] = (md["layers"][-1][0].astype(np.float64), md["layers"][-1][1].astype(np.float64))
    segs = O.ray_segments(td, o, d, M)
    so = O.emit_samples(segs, o, d, O.jitter_for_segments(seed, segs))

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))

    out = {"rays": R, "samples": int(segs["n"].sum())}
    for name, f_, m_ in (("vs_bf16_params", fd_b, md_b), ("vs_fp32_params", fd, md)):
        ref = O.project_forward(f_, m_, td, so, R, np.float64)
        g = O.project_backward(f_, m_, td, so, R, gi, np.float64)
        pg = np.concatenate([geo.planes[k].grad.cpu().numpy().ravel() for k in range(3)])
        pr = np.concatenate([g["planes"][k].ravel() for k in range(3)])
        lg = np.concatenate([geo.lines[k].grad.cpu().numpy().ravel() for k in range(3)])
        lr = np.concatenate([g["lines"][k].ravel() for k in range(3)])
        dg = np.concatenate([x.grad.cpu().numpy().ravel() for x in list(geo.decoder_weight) + list(geo.decoder_bias)])
        dr = np.concatenate([x.ravel() for x in list(g["W"]) + list(g["b"])])
        out[name] = {"image": rel(img.detach().cpu().numpy(), ref), "plane_grad": rel(pg, pr),
                     "line_grad": rel(lg, lr), "decoder_grad": rel(dg, dr)}
    return out


def make_host_shapes(R):
    """The host tensors one e2e step copies: origin and direction [R, 3] and
    the target [1, R], float32."""
    import torch

    return [torch.empty(R, 3), torch.empty(R, 3), torch.empty(1, R)]


def run_profile(args):
    """--profile-steps: the BF16 form's fused forward and backward on one
    batch of the workload, repeated, for ncu."""
    import torch

    import adaptivetensordf_b200 as ab
    from adaptivetensordf_b200 import synthetic as syn

    cfg = dataclasses.replace(workload_config(args.workload), rays_per_batch=args.rays)
    tree, dev, _, nseg, nsamp = prepare_workload(cfg, args.rays, 0, nb=1)
    geo = syn.make_geometry(tree, cfg.channels, cfg.grid, cfg.lines(), cfg.hidden, seed=1003)
    geo.precision = "bf16"
    geo.RefreshLowPrecision()
    o, d, _ = dev[0]
    rays = ab.RayList(o, d)
    for k in range(args.profile_steps):
        img = geo.ProjectRays(tree, rays, cfg.max_samples_per_node, 1 + k)
        img.sum().backward()
        for prm in syn.parameters(geo):
            prm.grad = None
    torch.cuda.synchronize()
    geo.CheckErrors()
    print(json.dumps({"profile_steps": args.profile_steps, "workload": cfg.name, "rays": args.rays,
                      "segments": nseg, "samples": nsamp}), flush=True)


def main():
    args = parse()
    if args.profile_steps:
        run_profile(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
