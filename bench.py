#!/usr/bin/env python
"""MLEM throughput on one B200 (or N, views sharded) -- one JSON line on rank 0.

Workload: 256^3 FP32 volume of 0.25 mm voxels, 360 views of a 512x512
detector of 0.5 mm pixels (source-isocentre 500 mm, source-detector 800 mm),
seeded 40-ellipsoid phantom, Poisson noise at I0 = 1e5.  A step is one MLEM
iteration: forward projection of all 360 views with the ratio g / Hf fused
in, then back projection of the ratios with the update f <- f*Ht/sens fused
in.  Inputs (the 377 MB measured sinogram and the ratio sinogram) are larger
than the L2 cache, so no flush is inserted between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl recon_b200|reference]

--impl reference times the reference's own CPU path: its Siddon kernel
sources compiled for the host (oracle/_ref/libref_cpu.so), run with its
step-synchronous per-view structure on all host threads, on a bounded sample
of views of one MLEM iteration, extrapolated to iterations per second.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MLEM iters/s & ray-voxel isects/s, batched vs plain on 1 B200 at <=1e-4 rel L2 vs FP64"
UNIT = "MLEM iter/s"
WORKLOAD = "plain_gpu_256cube_360x512x512"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="recon_b200", choices=["recon_b200", "reference"])
    ap.add_argument("--sum", default="kahan", choices=["kahan", "plain"])
    ap.add_argument("--sino", default="f32", choices=["f32", "bf16"],
                    help="storage of the measured and ratio sinograms (FP32 accumulation either way)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-baseline-steps", type=int, default=24)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-vs-plain leg")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the batched-vs-plain leg and print it as the JSON line")
    ap.add_argument("--no-voxel", action="store_true", help="skip the voxel-driven back projector leg")
    ap.add_argument("--no-compat", action="store_true", help="skip the COMPAT (reference arithmetic) leg")
    ap.add_argument("--large36", choices=["both", "whole", "blocks"],
                    help="only the 512^3 / 1024x768 / 36-view forward and back step, with the column forward "
                         "projector walking the volume whole (fp_block -1), in xy blocks (AUTO) or both; "
                         "one JSON line per design")
    ap.add_argument("--batched-problems", type=int, default=48)
    ap.add_argument("--batched-iters", type=int, default=20)
    return ap.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """SM clock and throttle-reason samples while the timed region runs: read
    through NVML every 10 ms (a timed region of ~0.1 s gives about ten), or
    from nvidia-smi every 200 ms where NVML cannot be loaded.  Reads only."""

    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.active",
              "clocks_event_reasons.hw_slowdown", "clocks_event_reasons.hw_thermal_slowdown",
              "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.lines: list[str] = []
        self.samples: list[tuple[float, float, int]] = []  # NVML: (sm MHz, max sm MHz, reason bits)
        self.proc = None
        self.nvml = None
        self.done = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.bits = [getattr(pynvml, "nvmlClocksEventReason" + n) for n in
                         ("HwSlowdown", "HwThermalSlowdown", "SwThermalSlowdown", "SwPowerCap")]
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), "--query-gpu=" + ",".join(self.FIELDS),
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _poll(self):
        nv, h = self.nvml, self.handle
        while not self.done.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), int(rs)))
            except Exception:
                return
            self.done.wait(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        sm, mx, reasons = [], [], set()
        if self.nvml is not None:
            self.done.set()
            self.t.join(timeout=5)
            for a, b, rs in self.samples:
                sm.append(a)
                mx.append(b)
                reasons.update(nm for nm, bit in zip(self.NAMES, self.bits) if rs & bit)
            source = "nvml, 10 ms"
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            for ln in self.lines:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) < len(self.FIELDS):
                    continue
                try:
                    sm.append(float(parts[0]))
                    mx.append(float(parts[1]))
                except ValueError:
                    continue
                for nm, val in zip(self.NAMES, parts[4:8]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
            source = "nvidia-smi, 200 ms"
        else:
            return None
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "source": source}


def gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v for v in vis.split(",") if v.strip()]
        if local_rank < len(ids) and ids[local_rank].strip().isdigit():
            return int(ids[local_rank])
    return local_rank


DATA = ("synthetic (seeded 40-ellipsoid phantom in a 0.02/mm cylinder, Poisson noise I0=1e5 drawn view by view "
        "from seed*100000+view)")


def workload_config(args, world: int = 1) -> dict:
    """The `config` of both arms' JSON lines."""
    return {"workload": WORKLOAD, "volume": [256, 256, 256], "voxel_mm": 0.25, "views": 360,
            "detector": [512, 512], "pixel_mm": 0.5, "arith": "exact", "sum": args.sum, "sino": args.sino,
            "parallelism": f"views/{world}" if world > 1 else "single",
            "l2": "no flush: per-step inputs (377 MB sinogram + 377 MB ratio) exceed the 126 MB L2"}


def make_problem(cfg, device):
    """Phantom and noisy measurement for the workload (recon_b200.phantom.workload):
    the numpy phantom, projected by the EXACT projector on the device, Poisson
    noise view by view on the host."""
    from recon_b200.phantom import workload

    return workload(cfg, device)


TRAFFIC_PROFILE = "profiles/exact_fp_column_bp_mirror_plain256_360v_512.md"
ACCURACY_PROFILE = "profiles/accuracy_plain256_360v_512.md"


def measured_traffic() -> dict:
    """DRAM bytes per forward / back projection of the bench workload, from the
    committed ncu summary (line `traffic-per-launch: fp=<bytes> bp=<bytes>`)."""
    import re

    try:
        text = open(os.path.join(ROOT, TRAFFIC_PROFILE)).read()
    except OSError:
        return {}
    m = re.search(r"traffic-per-launch:\s*fp=(\d+)\s+bp=(\d+)", text)
    return {"fp": int(m.group(1)), "bp": int(m.group(2))} if m else {}


def measured_accuracy() -> dict | None:
    """Error of this workload against FP64, as the GPU accuracy test measured it
    (committed summary, line `accuracy: {json}`): relative L2 of one MLEM update
    against the FP64 update of the same image on the central 16 slices, at
    iterations 1, 10 and 20, and the projectors' pair counts."""
    import re

    try:
        text = open(os.path.join(ROOT, ACCURACY_PROFILE)).read()
    except OSError:
        return None
    m = re.search(r"^accuracy:\s*(\{.*\})\s*$", text, re.M)
    if not m:
        return None
    d = json.loads(m.group(1))
    d["source"] = ACCURACY_PROFILE
    return d


def adjoint_check(P, seed: int = 7) -> float:
    """|<Ax, y> - <x, A^T y>| / |<Ax, y>| for random x, y on the plan's own
    projector pair (FP64 dot products of the FP32 results), measured in this run."""
    import torch

    gen = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.rand(P.shape_vol, device="cuda", generator=gen)
    y = torch.rand((P.nproj, P.nv, P.nu), device="cuda", generator=gen)
    lhs = torch.dot(P.fp_views(x).double().ravel(), y.double().ravel()).item()
    rhs = torch.dot(x.double().ravel(), P.bp_views(y).double().ravel()).item()
    return abs(lhs - rhs) / abs(lhs)


def shard_problems(work: list[float], world: int) -> list[list[int]]:
    """Problems per rank: largest first, each to the least-loaded rank."""
    out: list[list[int]] = [[] for _ in range(world)]
    load = [0.0] * world
    for p in sorted(range(len(work)), key=lambda i: -work[i]):
        r = min(range(world), key=lambda j: load[j])
        out[r].append(p)
        load[r] += work[p]
    return out


def batched_leg(device, n_prob: int, iters: int, opts, rank: int = 0, world: int = 1):
    """48 generated problems of uneven sizes: `iters` graph-captured MLEM
    iterations of all of them through one Batch, against the same iterations
    as sequential per-problem Plan.mlem calls (sensitivities cached in both).
    Both arms produce bit-identical images (checked here).  With several
    ranks the problems are sharded by rank (no communication) and the times
    are the max over ranks."""
    import torch

    from recon_b200 import SIDDON_BP_GATHER, SIDDON_BP_TUNED, Batch, Options, Plan
    from recon_b200.configs import batched_problems
    from recon_b200.phantom import noisy, phantom

    # both arms choose each problem's back projector by measurement
    # (SIDDON_BP_TUNED, kept per geometry, so both make the same choice)
    opts = Options(sum=opts.sum, sino=opts.sino, device=opts.device, siddon_bp=SIDDON_BP_TUNED)
    all_cfgs = batched_problems(n_prob, seed=4, iters=iters)
    work = [float(c["NumProj"]) * c["AxPixels"] * c["TAxPixels"] * (c["Xdim"] + c["Ydim"] + c["Zdim"])
            for c in all_cfgs]
    mine = shard_problems(work, world)[rank]
    cfgs = [all_cfgs[p] for p in mine]
    plans = [Plan(c, opts) for c in cfgs]
    gs = []
    for c, P in zip(cfgs, plans):
        vol = torch.from_numpy(phantom(c)).to(device)
        gs.append(noisy(P.fp_views(vol), c["I0"], c["seed"]))
        del vol
    for P in plans:
        P.mlem_prepare()
    B = Batch(cfgs, opts)
    fb = B.new_volumes()
    B.mlem(gs, 1, fb)  # autotune + graph capture
    fp = [P.new_volume() for P in plans]
    for P, g, f in zip(plans, gs, fp):
        P.mlem(g, 1, f)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    B.mlem(gs, iters, fb)
    e1.record()
    for P, g, f in zip(plans, gs, fp):
        P.mlem(g, iters, f)
    e2.record()
    torch.cuda.synchronize()
    t_batch = e0.elapsed_time(e1) * 1e-3
    t_plain = e1.elapsed_time(e2) * 1e-3
    same = all(torch.equal(a.view(torch.int32), b.view(torch.int32)) for a, b in zip(fb, fp))
    isects_each = [P.count_intersections() for P in plans]
    isects = sum(isects_each)
    n_gather = sum(1 for P in plans if P.siddon_bp == SIDDON_BP_GATHER)
    # each problem's forward step and back projection timed alone (after the
    # comparison above): what the batch can at best add up to
    alone = []
    for P, g, f in zip(plans, gs, fp):
        P.mlem_forward(g, f)
        P.mlem_backward_update(f)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        P.mlem_forward(g, f)
        e[1].record()
        P.mlem_backward_update(f)
        e[2].record()
        torch.cuda.synchronize()
        alone.append((e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])))
    bins = []
    for lo, hi in ((0, 30), (30, 60), (60, 120), (120, None)):
        sel = [k for k, c in enumerate(cfgs)
               if lo <= isects_each[k] / (c["Xdim"] * c["Ydim"] * c["NumProj"]) < (hi or float("inf"))]
        if sel:
            n_is = sum(isects_each[k] for k in sel)
            bins.append({"isects_per_column_view": [lo, hi], "problems": len(sel),
                         "fp_isects_per_s": n_is / (1e-3 * sum(alone[k][0] for k in sel)),
                         "bp_isects_per_s": n_is / (1e-3 * sum(alone[k][1] for k in sel))})
    alone_s = 1e-3 * sum(a + b for a, b in alone)
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([t_batch, t_plain], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_batch, t_plain = float(t[0]), float(t[1])
        q = torch.tensor([isects, 1 if same else 0], dtype=torch.int64, device=device)
        dist.all_reduce(q, op=dist.ReduceOp.SUM)
        isects, same = int(q[0]), int(q[1]) == world
    cfgs = all_cfgs
    vox = [int(c["Xdim"]) * int(c["Ydim"]) * int(c["Zdim"]) for c in cfgs]
    return {
        "problems": n_prob, "iters": iters,
        "batched_iter_s": n_prob * iters / t_batch, "plain_iter_s": n_prob * iters / t_plain,
        "speedup": t_plain / t_batch, "batched_isects_per_s": 2.0 * isects * iters / t_batch,
        "plain_isects_per_s": 2.0 * isects * iters / t_plain, "bitwise_equal": bool(same),
        "back_projectors": {"gather": n_gather, "ray": len(plans) - n_gather, "choice": "measured per geometry"},
        "forward_rows_per_cta": {str(r): sum(1 for P in plans if P.column_rows == r) for r in (0, 32, 64, 128)},
        "alone": {"serial_iter_s": len(plans) / alone_s, "isects_per_s": 2.0 * isects / alone_s, "by_work": bins,
                  "note": "each problem's forward step and back projection timed alone on this rank"},
        "sharding": f"problems by rank over {world} GPUs" if world > 1 else "single GPU",
        "config": {"workload": f"batched_{n_prob}_seed4", "voxels_min_max": [min(vox), max(vox)],
                   "views_min_max": [min(int(c["NumProj"]) for c in cfgs), max(int(c["NumProj"]) for c in cfgs)],
                   "isects_per_pass": isects},
    }


def voxel_leg(cfg, g, steps: int, warmup: int, device_index: int):
    """The same MLEM iteration with the voxel-driven back projector
    (geometric mode: FP32 bilinear taps, gathered per voxel column) in place
    of the Siddon one: Siddon forward projection with the plain ratio, then
    the voxel-driven back projection with the update fused in."""
    import torch

    from recon_b200 import BP_VOXEL, VOXEL_GEOMETRIC, Options, Plan

    P = Plan(cfg, Options(bp=BP_VOXEL, voxel_mode=VOXEL_GEOMETRIC, device=device_index))
    P.mlem_prepare()
    f = P.new_volume(1.0)
    for _ in range(warmup):
        P.mlem_iteration(g, f)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(steps):
        P.mlem_iteration(g, f)
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / steps
    return {"value": 1e3 / ms, "unit": UNIT, "ms_per_step": ms, "steps": steps, "warmup": warmup,
            "back_projector": "voxel-driven, FP32 bilinear taps gathered per voxel column (geometric mode)"}


def compat_leg(cfg, g, device_index: int, budget_s: float = 10.0):
    """The drop-in default path on the same workload: COMPAT arithmetic (the
    reference's FP32 Siddon traversal, hf_siddon_class.hpp:44-47 defaults),
    one thread per ray, int64 fixed-point scatter per view.  One untimed
    iteration, then iterations timed one by one with CUDA events until
    `budget_s` of timed work or 5 iterations."""
    import torch

    from recon_b200 import ARITH_COMPAT, Options, Plan

    P = Plan(cfg, Options(arith=ARITH_COMPAT, device=device_index))
    P.mlem_prepare()
    f = P.new_volume(1.0)
    P.mlem_iteration(g, f)
    times = []
    while len(times) < 5 and sum(times) < budget_s * 1e3:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        P.mlem_iteration(g, f)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    ms = sum(times) / len(times)
    P.close()
    return {"value": 1e3 / ms, "unit": UNIT, "ms_per_step": ms, "steps": len(times), "warmup": 1,
            "arithmetic": "COMPAT (the reference's FP32 traversal; bit-exact per ray)"}


def large36_leg(which: str, device_index: int):
    """512^3 volume of 0.125 mm, 1024 x 768 detector of 0.25 mm, 36 consecutive views
    at 0.5 deg, a seeded random volume in [0, 0.05): one MLEM forward step and one
    back projection with the update, best of 3 by CUDA events after 3 warm-up
    iterations, for the column forward projector over the whole volume and / or
    in xy blocks.  With both, the pair counts and the two images after the 4
    iterations are compared."""
    import torch

    from recon_b200 import PROJECTOR_FORWARD, Options, Plan
    from recon_b200.configs import LARGE, scaled

    cfg = scaled(LARGE, NumProj=36, DeltaAng=0.5)
    gen = torch.Generator("cuda").manual_seed(1)
    vol = torch.rand((512, 512, 512), device="cuda", generator=gen) * 0.05
    sides = {"whole": [-1], "blocks": [0], "both": [-1, 0]}[which]
    images = []
    for side in sides:
        P = Plan(cfg, Options(fp_block=side, device=device_index))
        g = P.fp_views(vol)
        P.mlem_prepare()
        f = P.new_volume(1.0)
        for _ in range(3):
            P.mlem_forward(g, f)
            P.mlem_backward_update(f)
        torch.cuda.synchronize()
        ts = []
        for _ in range(3):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            e[0].record()
            P.mlem_forward(g, f)
            e[1].record()
            P.mlem_backward_update(f)
            e[2].record()
            torch.cuda.synchronize()
            ts.append((e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])))
        line = {"workload": "large_512cube_36x1024x768", "fp_block": side, "forward_projector": P.forward_projector,
                "forward_ms": min(t[0] for t in ts), "backward_ms": min(t[1] for t in ts)}
        if which == "both":
            line["pairs_forward"] = P.count_projector_pairs(PROJECTOR_FORWARD)
            line["isects"] = P.count_intersections()
            images.append(f.double())
        print(json.dumps(line), flush=True)
        del P, g, f
        torch.cuda.empty_cache()
    if len(images) == 2:
        a, b = images
        print(json.dumps({"image_rel_l2_blocks_vs_whole_after_4_iterations": ((a - b).norm() / a.norm()).item()}))


def ref_view_seconds(R, O, geo, cfg, view, steps, f, gview, ht):
    """Seconds for one view of one MLEM iteration with the reference's
    step-synchronous kernels built for the host, from a timed prefix of
    `steps` of its loopN step launches (each step launches the same kernels
    over all rays and the whole volume, so a view costs (loopN + 1) /
    (steps + 1) times the prefix)."""
    import numpy as np

    ang = float(np.float32(view) * np.float32(cfg["DeltaAng"]))
    loopN = O.c_loopN(geo, ang)
    s = min(steps, loopN)
    t0 = time.perf_counter()
    R.ref_cpu_mlem_view_steps(geo, ang, s, f, gview, ht)
    dt = time.perf_counter() - t0
    return dt * (loopN + 1) / (s + 1), dt, loopN, s


def cpu_baseline(cfg, g_host, steps: int = 24):
    """The reference's kernels built for the host on one thread: one view of
    the first MLEM iteration (f = 1), extrapolated to iterations/s."""
    import numpy as np

    from oracle import oracle as O
    from recon_b200.configs import geom_dict

    R = O.ref_cpu()
    if R is None:
        return None
    R.ref_cpu_set_threads(1)
    geo = O.Geom.from_dict(geom_dict(cfg))
    f = np.ones(geo.nvox, np.float32)
    ht = np.zeros(geo.nvox, np.float32)
    n = int(cfg["NumProj"])
    view = n // 10
    t_view, dt, loopN, s = ref_view_seconds(R, O, geo, cfg, view, steps, f,
                                            np.ascontiguousarray(g_host[view].ravel()), ht)
    out = {"value": 1.0 / (t_view * n), "unit": UNIT, "cores": 1, "kind": "reference",
           "sample": f"view {view} of one MLEM iteration (FP + ratio + BP with the reference's step-synchronous "
                     f"kernels built for the host): the first {s} of its {loopN} step launches took {dt:.1f} s, "
                     f"scaled by (loopN+1)/(steps+1) to {t_view:.0f} s/view and by {n} views"}
    # the per-ray FP64 Siddon oracle (one thread per view group), for scale
    vol = np.ones(geo.nvox)
    fp64 = {}
    cores = os.cpu_count() or 1
    for label, threads, nv in (("1_core", 1, 4), ("all_cores", cores, max(4, 2 * cores))):
        t0 = time.perf_counter()
        sino = O.x_fp_all(geo, nv, 360.0 / nv, vol, threads)
        O.x_bp_all(geo, nv, 360.0 / nv, sino, threads)
        fp64[label] = nv / ((time.perf_counter() - t0) * n)
    out["fp64_oracle"] = {"iter_s_1_core": fp64["1_core"], "iter_s_all_cores": fp64["all_cores"],
                          "cores": cores, "unit": UNIT,
                          "sample": f"FP + BP with the per-ray FP64 Siddon oracle of 4 evenly spaced views on one "
                                    f"thread and of max(4, 2 x cores) on all, extrapolated to {n} views"}
    return out


def reference_gpu_leg(O, geo, cfg, vol, gviews: dict) -> dict | None:
    """The reference's own CUDA implementation on this GPU (its sources built for
    sm_100a, oracle/_ref/libref_gpu.so), driven through its forward / backward
    classes as its MLEM loop drives them per view (a_calc_initial_limits with
    its blocking step-count read-back, the step-synchronous kernels, one view
    in and one image out): FP then BP of the sampled views, extrapolated to the
    360 views of an iteration.  The elementwise ratio and update kernels are
    left out (a small part).  None when that build is missing."""
    import numpy as np

    R = O.ref_gpu()
    if R is None:
        return None
    import torch

    if not torch.cuda.is_available():  # the reference exits the process on a CUDA error
        return {"unavailable": "no CUDA device"}
    n = int(cfg["NumProj"])
    dang = np.float32(cfg["DeltaAng"])
    vol32 = vol.astype(np.float32)
    img = np.zeros(geo.npix, np.float32)
    bp = np.zeros(geo.nvox, np.float32)
    R.ref_gpu_fp_view(geo, 0.0, vol32, img)  # context and module load
    t_fp = t_bp = 0.0
    views = sorted(gviews)
    for v in views:
        ang = float(np.float32(v) * dang)
        t0 = time.perf_counter()
        R.ref_gpu_fp_view(geo, ang, vol32, img)
        t1 = time.perf_counter()
        R.ref_gpu_bp_view(geo, ang, gviews[v], bp)
        t2 = time.perf_counter()
        t_fp += t1 - t0
        t_bp += t2 - t1
    per_view = (t_fp + t_bp) / len(views)
    return {"value": 1.0 / (per_view * n), "unit": UNIT, "s_per_iteration": per_view * n,
            "fp_s_per_view": t_fp / len(views), "bp_s_per_view": t_bp / len(views),
            "sample": f"views {views}: forward and back projection each through the reference's classes, "
                      f"extrapolated x{n}"}


def small_full_iteration(R, O, threads: int, prefix: int) -> dict:
    """The extrapolation above, checked where it can be measured in full: one
    MLEM iteration of the 64^3 / 90-view / 128^2 workload (configs.CPU_SMALL)
    with the reference's step-synchronous kernels built for the host, every
    view run to its last step, against the same views predicted from their
    first `prefix` step launches."""
    import numpy as np

    from recon_b200.configs import CPU_SMALL, geom_dict

    cfg = dict(CPU_SMALL)
    geo = O.Geom.from_dict(geom_dict(cfg))
    n = int(cfg["NumProj"])
    rng = np.random.default_rng(1)
    f = np.ones(geo.nvox, np.float32)
    ht = np.zeros(geo.nvox, np.float32)
    full = predicted = 0.0
    for v in range(n):
        gview = rng.random(geo.npix).astype(np.float32)
        predicted += ref_view_seconds(R, O, geo, cfg, v, prefix, f, gview, ht)[0]
        full += ref_view_seconds(R, O, geo, cfg, v, 1 << 30, f, gview, ht)[1]
    return {"workload": "cpu_small_64cube_90x128x128", "threads": threads, "measured_s_per_iteration": full,
            "predicted_s_per_iteration": predicted, "predicted_over_measured": predicted / full,
            "sample": f"every view of one MLEM iteration run to its last step, and predicted from its first "
                      f"{prefix} step launches"}


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    import numpy as np

    from recon_b200.configs import PLAIN_GPU, geom_dict

    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True}
    try:
        from oracle import oracle as O
    except Exception as e:  # pragma: no cover
        print(json.dumps({**base, "unavailable": f"checker package not importable: {e}"}))
        return
    R = O.ref_cpu()
    if R is None:
        print(json.dumps({**base, "unavailable": "reference host build oracle/_ref/libref_cpu.so missing"}))
        return
    cfg = dict(PLAIN_GPU)
    threads = os.cpu_count() or 1
    R.ref_cpu_set_threads(threads)
    geo = O.Geom.from_dict(geom_dict(cfg))
    from recon_b200.phantom import noisy, phantom

    vol = phantom(cfg).astype(np.float64).ravel()
    n = int(cfg["NumProj"])
    dang = np.float32(cfg["DeltaAng"])
    nsample = max(1, args.steps + args.warmup)
    views = [int(round(k * n / nsample)) % n for k in range(nsample)]
    # the GPU arm's inputs for these views: the same phantom, projected (here in
    # FP64, there by the FP32 EXACT projector: equal to ~1e-7 relative) and the
    # same Poisson draws (noisy_views: view n from seed * 100000 + n)
    gpu_views = [k * n // 8 for k in range(8)]  # the reference's CUDA build: 8 evenly spaced views
    gviews = {}
    for v in sorted(set(views) | set(gpu_views)):
        img = np.zeros(geo.npix)
        O.lib().orc_x_fp_view(geo, float(np.float32(v) * dang), vol, img)
        gviews[v] = noisy(img, cfg["I0"], cfg["seed"] * 100000 + v).astype(np.float32)
    f = np.ones(geo.nvox, np.float32)
    ht = np.zeros(geo.nvox, np.float32)
    times, sample_s = [], []
    prefix = 48
    for k, v in enumerate(views):
        t_view, dt, _, _ = ref_view_seconds(R, O, geo, cfg, v, prefix, f, gviews[v], ht)
        if k >= args.warmup:
            times.append(t_view)
            sample_s.append(dt)
    tv = sum(times) / len(times)
    value = 1.0 / (tv * n)
    sample = (f"{len(times)} timed views (+{args.warmup} warm-up) of one MLEM iteration of the 256^3 / 360-view "
              f"workload with the reference's step-synchronous kernels built for the host on {threads} threads; "
              f"each view timed on the first {prefix} of its step launches and scaled by (loopN+1)/(steps+1) "
              f"(mean {tv:.1f} s/view), extrapolated x{n}")
    out = {
        **base, "value": value, "n_gpus": world, "steps": len(times), "warmup": args.warmup,
        # a step is one sampled view's prefix of step launches: what was timed
        "ms_per_step": 1e3 * sum(sample_s) / len(sample_s),
        "extrapolated_ms_per_iteration": tv * n * 1e3,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": DATA,
        "config": workload_config(args, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        rg = reference_gpu_leg(O, geo, cfg, vol, {v: gviews[v] for v in gpu_views})
    except Exception as e:  # pragma: no cover
        rg = {"error": str(e)}
    if rg is not None:
        out["reference_gpu"] = rg
    out["extrapolation_check"] = small_full_iteration(R, O, threads, prefix)
    print(json.dumps(out))


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    from recon_b200 import (FP_COLUMN_BLOCKS, FP_COLUMNS, SIDDON_BP_GATHER, SINO_BF16, SINO_F32, SUM_KAHAN, SUM_PLAIN,
                            Options, Plan)
    from recon_b200.configs import PLAIN_GPU
    from recon_b200.sharding import sharded_mlem_iteration, view_range

    world, rank, local = dist_env()
    if args.large36:
        torch.cuda.set_device(local)
        large36_leg(args.large36, local)
        return
    if args.batched_only:
        torch.cuda.set_device(local)
        opts = Options(sum=SUM_KAHAN if args.sum == "kahan" else SUM_PLAIN, device=local)
        leg = batched_leg(torch.device("cuda", local), args.batched_problems, args.batched_iters, opts)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": leg["batched_iter_s"], "unit": "MLEM iter/s (problem-iterations)",
                              "n_gpus": 1, "higher_is_better": True, "batched": leg}))
        return
    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    cfg = dict(PLAIN_GPU)
    opts = Options(sum=SUM_KAHAN if args.sum == "kahan" else SUM_PLAIN,
                   sino=SINO_BF16 if args.sino == "bf16" else SINO_F32, device=local)
    vol, g = make_problem(cfg, device)
    if args.sino == "bf16":
        g = g.to(torch.bfloat16)
    P = Plan(cfg, opts)
    nviews = int(cfg["NumProj"])
    isects = P.count_intersections()
    P.mlem_prepare()
    f = P.new_volume(1.0)
    ht = P.new_volume(0.0)
    if P.quarter_sets:  # a rank's views: the same base range of each quarter (sharded_mlem_iteration)
        qf, qc = view_range(nviews // 4, rank, world)
        ranges = [(qf + r * (nviews // 4), qc) for r in range(4)]
    else:
        ranges = [view_range(nviews, rank, world)]
    count = sum(c for _, c in ranges)
    npix = P.nu * P.nv
    nvox = f.numel()
    # kernels per step: the volume's copy (z-fastest for the column forward
    # projector, xy-transposed for the ray walk) + the forward kernel; the gather
    # back projector is one kernel (after the ratio's transpose into detector
    # columns where the ray walk wrote it row-major), the ray-driven one maxabs +
    # (ray + finish) per z-slab (both int64 accumulators of a slab in 64 MiB);
    # at N > 1 a separate update
    gather = P.siddon_bp == SIDDON_BP_GATHER
    columns = P.forward_projector in (FP_COLUMNS, FP_COLUMN_BLOCKS)
    mirror = P.mirror_pairs
    Z, Y, X = P.shape_vol
    depth = max(1, min(Z, (64 << 20) // (X * Y * 16)))
    slabs = -(-Z // depth)
    bp_launches = (1 if columns else 2) if gather else 1 + 2 * slabs

    def iteration(ev=None):
        if world == 1:
            if ev:
                ev[0].record()
            P.mlem_forward(g, f)
            if ev:
                ev[1].record()
            P.mlem_backward_update(f)
            if ev:
                ev[2].record()
        else:
            sharded_mlem_iteration(P, g, f, ht)

    for _ in range(args.warmup):
        iteration()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(gpu_index(local)) if rank == 0 else None
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    for k in range(args.steps):
        iteration(evs[k] if world == 1 else None)
    end.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    if world > 1:
        t = torch.tensor([ms], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    clk = clocks.stop() if clocks else None
    ms_step = ms / args.steps
    value = 1e3 / ms_step

    # end to end through the C ABI with host buffers: every step uploads the
    # measured sinogram from pinned memory (recon_upload_sinogram: the rows
    # some ray crossing the volume reaches, as one strided copy) and reads the
    # image back.  The upload of step k+1 (its own stream, into the other of
    # two device buffers) and the read-back of step k (a third stream) overlap
    # the compute of the neighbouring steps; the timed region ends after the
    # last read-back.
    g_host = g.cpu().pin_memory()
    f_host = torch.empty(f.shape, dtype=torch.float32).pin_memory()
    e2e = None
    if world > 1:
        # each rank uploads its own views of the sinogram, rank 0 reads the image back
        h2d = [0]

        def e2e_sharded():
            h2d[0] = sum(P.upload_sinogram(g_host, g, a, c) for a, c in ranges)
            iteration()
            if rank == 0:
                f_host.copy_(f, non_blocking=True)

        for _ in range(max(1, args.warmup)):
            e2e_sharded()
        torch.cuda.synchronize()
        dist.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            e2e_sharded()
        b.record()
        torch.cuda.synchronize()
        t = torch.tensor([a.elapsed_time(b)], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item()) / args.steps
        e2e = {"value": 1e3 / e2e_ms, "unit": UNIT,
               "h2d_bytes_per_step": h2d[0], "d2h_bytes_per_step": f.numel() * 4 if rank == 0 else 0,
               "h2d_of_full_sinogram": count * npix * g.element_size(),
               "pipeline": "each rank uploads its views, rank 0 reads the image back (not overlapped)"}
    if world == 1:
        comp = torch.cuda.current_stream()
        up_s, down_s = torch.cuda.Stream(), torch.cuda.Stream()
        gbufs = [torch.empty_like(g), torch.empty_like(g)]
        uploaded = [torch.cuda.Event(), torch.cuda.Event()]
        released = [torch.cuda.Event(), torch.cuda.Event()]  # forward projection done reading the buffer
        f_written, f_read = torch.cuda.Event(), torch.cuda.Event()
        h2d = [0]

        def e2e_step(k):
            b = k % 2
            up_s.wait_event(released[b])
            with torch.cuda.stream(up_s):
                h2d[0] = P.upload_sinogram(g_host, gbufs[b])
            uploaded[b].record(up_s)
            comp.wait_event(uploaded[b])
            P.mlem_forward(gbufs[b], f)
            released[b].record(comp)
            comp.wait_event(f_read)  # the previous read-back is done before f is updated
            P.mlem_backward_update(f)
            f_written.record(comp)
            down_s.wait_event(f_written)
            with torch.cuda.stream(down_s):
                f_host.copy_(f, non_blocking=True)
            f_read.record(down_s)

        for k in range(max(1, args.warmup)):
            e2e_step(k)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(comp)
        for k in range(args.steps):
            e2e_step(k)
        comp.wait_event(f_read)
        b.record(comp)
        torch.cuda.synchronize()
        e2e_ms = a.elapsed_time(b) / args.steps
        e2e = {"value": 1e3 / e2e_ms, "unit": UNIT, "h2d_bytes_per_step": h2d[0],
               "d2h_bytes_per_step": f.numel() * 4, "h2d_of_full_sinogram": g.numel() * g.element_size(),
               "pipeline": "H2D of step k+1 (the detector rows the rays can reach) and D2H of step k on their "
                           "own streams, overlapping compute"}

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32" if args.sino == "f32" else "f32 (bf16 sinograms)",
        "data": DATA, "config": workload_config(args, world),
        "isects_per_pass": isects,
        "isects_per_s": 2.0 * isects * value,
        "gpu_launches": args.steps * (2 + bp_launches + (0 if world == 1 else 1)),
        "back_projector": "gather" if gather else "ray",
        "forward_projector": "detector columns" if columns else "ray walk",
        "ratio_layout": ("mirrored row pairs" if gather and mirror and columns and P.nv % 2 == 0 else
                         "detector columns" if gather else "rows"),
        "mirror_pairs": mirror,
        "quarter_turns": P.quarter_turns,
    }
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    if world == 1:
        t_fp = sum(e[0].elapsed_time(e[1]) for e in evs) / args.steps
        t_bp = sum(e[1].elapsed_time(e[2]) for e in evs) / args.steps
        bytes_fp = 4.0 * isects + 4.0 * npix * nviews
        bytes_bp = 4.0 * isects + 12.0 * nvox
        traffic = measured_traffic()
        if t_bp >= t_fp:
            # mirrored row pairs where both projectors pair rows (even detector height,
            # detector-column forward projector)
            pairs = mirror and columns and P.nv % 2 == 0
            dom = (("back projection (bp_gather_quarter_kernel)" if pairs and P.quarter_turns else
                    "back projection (bp_gather_pairs_kernel)" if pairs else
                    "back projection (bp_gather_mirror_kernel)" if mirror else "back projection (bp_gather_kernel)")
                   if gather else
                   "back projection (maxabs + bp_ray_kernel per z-slab + bp_finish_kernel)", t_bp, bytes_bp,
                   traffic.get("bp"))
        else:
            dom = ("forward projection (to_zfast_kernel + fp_column_kernel)" if columns else
                   "forward projection (transpose_xy_kernel + fp_kernel)", t_fp, bytes_fp, traffic.get("fp"))
        ach = dom[2] / (dom[1] * 1e-3) / 1e9
        out["roofline"] = {"bound": "hbm", "kernel": dom[0], "achieved": ach, "peak": hbm, "unit": "GB/s",
                           "frac": ach / hbm, "peak_source": peak_src, "traffic": dom[3],
                           "traffic_source": TRAFFIC_PROFILE if dom[3] is not None else None,
                           "algorithmic_bytes_per_launch": dom[2], "launch_ms": dom[1]}
        if dom[3] is not None:
            # the DRAM bytes the kernel moves (ncu): most algorithmic bytes (4 per
            # intersection) are served from L1 / L2, so frac can pass 1 while DRAM idles
            out["roofline"]["dram_achieved"] = dom[3] / (dom[1] * 1e-3) / 1e9
            out["roofline"]["dram_frac"] = out["roofline"]["dram_achieved"] / hbm
        b_iter = 8.0 * isects + 4.0 * npix * nviews + 12.0 * nvox
        b_comp = 4.0 * npix * nviews + 12.0 * nvox  # the bytes no design avoids: g once, f and sens read, f written
        out["iteration_roofline"] = {"bytes_per_iteration": b_iter, "achieved_gbs": b_iter / (ms_step * 1e-3) / 1e9,
                                     "frac": b_iter / (ms_step * 1e-3) / 1e9 / hbm,
                                     "compulsory_bytes": b_comp,
                                     "compulsory_frac": b_comp / (ms_step * 1e-3) / 1e9 / hbm,
                                     "fp_ms": t_fp, "bp_ms": t_bp}
        # the sensitivity image: one back projection of w, computed once per plan (outside the iterations)
        sens = P.new_volume(0.0)
        P.sensitivity(sens)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s0.record()
        P.sensitivity(sens)
        s1.record()
        torch.cuda.synchronize()
        out["sensitivity_ms"] = s0.elapsed_time(s1)
        del sens
        if P.quarter_sets:
            # one rank's back projection when two ranks split the views: a quarter set
            # (half the base views of each quarter) against a contiguous half range
            def bp_ms(call):
                call()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                call()
                e1.record()
                torch.cuda.synchronize()
                return e0.elapsed_time(e1)

            q = nviews // 4
            P.mlem_forward(g, f)
            out["two_rank_split_bp_ms"] = {
                "quarter_set": bp_ms(lambda: P.mlem_backward_quarters(ht, 0, q // 2)),
                "contiguous_range": bp_ms(lambda: P.mlem_backward(ht, 0, 4 * (q // 2))),
                "views_per_rank": 4 * (q // 2)}
    out["e2e"] = e2e
    out["clocks"] = clk
    if world == 1:
        acc = measured_accuracy() or {}
        acc["adjoint_rel_this_run"] = adjoint_check(P)
        out["accuracy"] = acc
    if world == 1 and not args.no_cpu_baseline:
        try:
            out["cpu_baseline"] = cpu_baseline(cfg, g_host.numpy().reshape(nviews, P.nv, P.nu),
                                               args.cpu_baseline_steps)
        except Exception as e:  # pragma: no cover
            out["cpu_baseline"] = {"error": str(e)}
    if world == 1 and not args.no_voxel and args.sino == "f32":
        del P
        torch.cuda.empty_cache()
        out["voxel_bp"] = voxel_leg(cfg, g, max(3, args.steps // 4), args.warmup, local)
    if world == 1 and not args.no_compat and args.sino == "f32":
        torch.cuda.empty_cache()
        out["compat"] = compat_leg(cfg, g, local)
    if not args.no_batched:
        del g_host, f_host, g, vol
        torch.cuda.empty_cache()
        out["batched"] = batched_leg(device, args.batched_problems, args.batched_iters, opts, rank, world)
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
