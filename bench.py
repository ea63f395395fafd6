#!/usr/bin/env python
"""Benchmark: plane-sweep NCC throughput (Mpix*planes/s) and TGV2 ms/frame on one B200 per rank.

Workload (one step = one reference frame):
  640x480 reference view + 8 source views with 2-10 cm baselines (seeded
  ray-cast box room textured with 4-octave value noise), 256 planes uniform in
  inverse depth over [0.4, 8] m, 9x9 NCC with compensated FP32 moments, cost
  = 1 - mean NCC stored as a BF16 cost volume [256][480][640], winner-take-all
  argmin over the stored volume.  Per step: FP64 homographies on the device,
  the fused sweep, the WTA pass.  Throughput counts pixel x plane x view NCC
  evaluations: 640*480*256*8 = 629.1M per frame.
  TGV2 (reported beside it): refinement of the WTA depth to relative energy
  change 1e-4 (checked every 10 iterations, cap 500).

Inputs are resident in HBM when the timed region starts; L2 is flushed (a
256 MiB write) before every timed step, outside the step's CUDA events.  With
--gpus N every rank sweeps its own frame (seed + rank): weak scaling, no
data-path collective (frames are independent).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mvs|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "plane-sweep-cuda_b200"))

import numpy as np  # noqa: E402

METRIC = "Mpix·planes/s NCC sweep; ms/frame to TGV2 energy tol, warm-start vs plain"
UNIT = "Mpix*planes/s"
# per-launch DRAM traffic (bytes) of the dominant kernels, from one `ncu --set full` capture each
# of `python bench.py --steps 2 --warmup 3 --tgv-steps 1 --no-cpu-baseline --no-batch
# --no-warm-start --no-fusion --no-reference-gpu` (one launch, dram__bytes_read.sum +
# dram__bytes_write.sum; the TGV2 iteration also with --no-tgv-sparse, launch 51: ncu runs every
# launch with a cold L2, so that figure is the whole working set, which stays in L2 between the
# back-to-back iterations of a run)
NCU_TRAFFIC = {"sweep_aggregated_kernel": 51.70432e6 + 128.86656e6,
               "wta_volume_kernel": 157.294336e6 + 3.661312e6,
               "tgv2_iteration_kernel": 47.945216e6 + 0.405248e6}
# algorithmic FP32 operations per (pixel, plane, view) evaluation of the fused sweep: homography
# 15 (kernels.cu:31-44), bilinear 8 (kernels.cu:4-29), three running window moments 14
# (kernels.cu:187-235), NCC 10 (kernels.cu:46-64), running best 3 (kernels.cu:66-82)
SWEEP_OPS_PER_EVAL = 50
W, H, V, P, WIN = 640, 480, 8, 256, 9
SEED = 2


def peaks():
    try:
        with open(ROOT / "MEASURED_PEAKS.json") as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def wait_first(self, timeout=5.0):
        """Block until nvidia-smi has produced its first sample (or timeout)."""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.01)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, window=None):
        """Median SM clock, max clock and active throttle reasons of the samples
        taken inside `window` (host times), or of all samples when none fell
        inside it (the window is then reported as the whole loaded run)."""
        lines = [ln for t, ln in self.lines if window and window[0] <= t <= window[1]]
        where = "timed region"
        if not lines:
            lines = [ln for _, ln in self.lines]
            where = "whole bench run (all sections under load)"
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm),
                "window": where, "interval_ms": 20}


def make_frame(rank: int):
    from mvs_b200 import scenes
    fr, planes, win = scenes.config_full(seed=SEED + rank)
    assert fr.ref.shape == (H, W) and len(fr.srcs) == V and len(planes) == P and win == WIN
    return fr, planes


def cpu_reference_sample(fr, planes, n_planes_sample=4):
    """The reference's own sweep kernels compiled for the CPU (all host threads), on a
    bounded sample of the workload: the full frame and all views, every 64th plane."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle as po
    sample = planes[:: P // n_planes_sample][:n_planes_sample]
    poses = [(c.R, c.t) for c in fr.src_cams]
    if po.ref_lib() is not None:
        r = po.ref_sweep(fr.ref, fr.srcs, fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, poses, sample, WIN,
                         zfar=8.0)
        secs, kind, cores = r["seconds"], "reference", os.cpu_count()
    else:
        Hs = po.homographies(fr.ref_cam.K_1based, fr.ref_cam.R, fr.ref_cam.t, poses, sample, precision="f32")
        t0 = time.perf_counter()
        po.sweep(fr.ref, fr.srcs, Hs, sample, WIN, zfar=8.0, precision="f32")
        secs, kind, cores = time.perf_counter() - t0, "port", 1
    evals = W * H * V * len(sample)
    return evals / secs / 1e6, secs, kind, cores, f"640x480 frame, 8 views, {len(sample)} of the 256 planes, 9x9"


def run_reference(args):
    from mvs_b200 import dist
    rank, ws, _ = dist.world()
    if rank != 0:
        return 0
    fr, planes = make_frame(0)
    for _ in range(args.warmup):
        cpu_reference_sample(fr, planes)
    vals = [cpu_reference_sample(fr, planes) for _ in range(args.steps)]
    tput = statistics.mean(v[0] for v in vals)
    secs = statistics.mean(v[1] for v in vals)
    _, _, kind, cores, sample = vals[0]
    line = {"metric": METRIC, "value": tput, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": secs * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ray-cast box room)",
            "impl": "reference",
            "config": {"workload": "sweep: 640x480, 8 views, 256 inverse-depth planes over [0.4, 8] m, 9x9 NCC",
                       "sample_per_step": sample},
            "cpu_baseline": {"value": tput, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": tput, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference_gpu(fr, planes, dev, d_ref, d_srcs, wta_depth):
    """The reference's RunAlgorithm and TGV call sequences with its own kernels compiled for
    this GPU (oracle/_ref/libmvs_ref_gpu.so), beside this engine in the reference's arithmetic
    (per-view sweep, reference moments, the reference's float homographies) on the same frame."""
    import torch
    import mvs_b200 as M
    from mvs_b200 import hostmath as hm
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle as po
    if po.ref_gpu_lib() is None:
        return {"unavailable": "oracle/_ref/libmvs_ref_gpu.so was not built (needs the reference tree)"}
    K1 = np.float32(fr.ref_cam.K_1based)
    poses = [(np.float32(c.R), np.float32(c.t)) for c in fr.src_cams]
    Rref, tref = np.float32(fr.ref_cam.R), np.float32(fr.ref_cam.t)
    evals = W * H * P * V
    out = {"kernels": "the reference's kernels.cu / TGV2_kernels.cu, unchanged, nvcc sm_100a",
           "sweep": {}, "tgv2_500_iterations": {}}
    ms = []
    for k in range(2):
        _, t = po.ref_gpu_sweep(fr.ref, fr.srcs, K1, Rref, tref, poses, planes, WIN, 8.0)
        if t < 0:
            return {"unavailable": "a CUDA error in the reference's kernels"}
        if k:
            ms.append(t)
    out["sweep"]["reference_ms"] = min(ms)
    out["sweep"]["reference_value"] = evals / (min(ms) / 1e3) / 1e6
    # this engine, reference arithmetic: per-view sweep + combine, reference float homographies
    iK = hm.inv3_f32(K1)
    rel = [hm.relative_f32(fr.ref_cam.R, fr.ref_cam.t, c.R, c.t) for c in fr.src_cams]
    Hh = np.stack([np.stack([hm.homography_f32(K1, iK, r[0], r[1], np.float32(d)).reshape(9) for d in planes])
                   for r in rel]).astype(np.float32)
    d_H = torch.from_numpy(Hh.reshape(-1)).to(dev)
    d_planes = torch.from_numpy(planes).to(dev)
    desc = M.sweep_desc(W, H, V, P, WIN, M.MOMENTS_REFERENCE, M.SWEEP_PER_VIEW, 1e-4, 0.5, 8.0)
    depth = torch.empty((H, W), device=dev)
    ws = torch.empty(M.sweep_workspace_bytes(desc) // 8 + 1, dtype=torch.int64, device=dev)
    em = []
    for k in range(4):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        M.sweep(desc, d_ref, d_srcs, d_H, d_planes, depth, None, None, None, ws)
        b.record()
        torch.cuda.synchronize()
        if k:
            em.append(a.elapsed_time(b))
    out["sweep"]["this_engine_reference_arithmetic_ms"] = min(em)
    out["sweep"]["this_engine_reference_arithmetic_value"] = evals / (min(em) / 1e3) / 1e6
    out["sweep"]["speedup"] = min(ms) / min(em)
    if wta_depth is not None:
        u0 = wta_depth.cpu().numpy()
        _, t = po.ref_gpu_tgv(fr.ref, fr.srcs, K1, Rref, tref, poses, 500, 1, u_init=u0)
        out["tgv2_500_iterations"]["reference_ms"] = t
        Kf, Rs = K1.reshape(9), np.stack([r[0].reshape(9) for r in rel])
        ts = np.stack([r[1] for r in rel])
        prm = M.tgv2_params(niters=500, warps=1)
        u = torch.empty((H, W), device=dev)
        tw = torch.empty(M.tgv2_workspace_bytes(W, H, V) // 8 + 1, dtype=torch.int64, device=dev)
        tm = []
        for k in range(3):
            u.copy_(wta_depth)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            M.tgv2_run(d_ref, d_srcs, Kf, iK.reshape(9), Rs, ts, prm, u, u_from_input=True, workspace=tw)
            b.record()
            torch.cuda.synchronize()
            if k:
                tm.append(a.elapsed_time(b))
        out["tgv2_500_iterations"]["this_engine_ms"] = min(tm)
        out["tgv2_500_iterations"]["speedup"] = t / min(tm)
    return out


SPARSE_ITERS = 200
SPARSE_BYTES_PER_PIXEL_ITERATION = 84   # u, v(2), p(2), q(3) read and written + T(3), weight, Ds read; fp32


def run_tgv_sparse(fr, dev, d_ref, wta_depth, peak_gbs, reference_gpu):
    """PlaneSweep::TGVdenoiseFromSparse on the bench frame: TGV2 from the WTA depth towards a
    seeded 5% sample of the true depth, 200 iterations, one fused launch per iteration; beside
    it the reference's own three launches per iteration on this GPU."""
    import torch
    import mvs_b200 as M
    rng = np.random.default_rng(77)
    gt = fr.depth_gt
    sparse = np.where(rng.random(gt.shape) < 0.05, gt, 0).astype(np.float32)
    d_sp = torch.from_numpy(sparse).to(dev)
    out = torch.empty((H, W), device=dev)
    ws = torch.empty(M.tgv2_sparse_workspace_bytes(W, H) // 8 + 1, dtype=torch.int64, device=dev)
    times = {}
    for iters in (0, SPARSE_ITERS):
        tm = []
        for k in range(4):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            M.tgv2_sparse(d_ref, wta_depth, d_sp, 8.0, out, ws, iters)
            b.record()
            torch.cuda.synchronize()
            if k:
                tm.append(a.elapsed_time(b))
        times[iters] = min(tm)
    per_it = (times[SPARSE_ITERS] - times[0]) / SPARSE_ITERS
    res = {"workload": f"640x480, {SPARSE_ITERS} iterations, 5% of the pixels sampled, from the WTA depth",
           "ms": times[SPARSE_ITERS], "ms_per_iteration": per_it,
           "roofline": {"bound": "hbm", "achieved": SPARSE_BYTES_PER_PIXEL_ITERATION * W * H / (per_it / 1e3) / 1e9,
                        "peak": peak_gbs, "unit": "GB/s",
                        "bytes_per_pixel_iteration": SPARSE_BYTES_PER_PIXEL_ITERATION,
                        "note": "the 25.8 MB state is L2-resident across iterations"}}
    res["roofline"]["frac"] = res["roofline"]["achieved"] / peak_gbs
    if reference_gpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import pyoracle as po
        if po.ref_gpu_lib() is not None:
            u0 = wta_depth.cpu().numpy()
            rt = []
            for k in range(2):
                ru, t = po.ref_gpu_tgv_sparse(fr.ref, u0, sparse, 8.0, SPARSE_ITERS)
                rt.append(t)
            mine = out.cpu().numpy()
            rel = np.abs(mine - ru) / np.maximum(np.abs(ru), 1e-30)
            res["reference_gpu_ms"] = rt[-1]
            res["speedup_vs_reference_gpu"] = rt[-1] / times[SPARSE_ITERS]
            # the reference's GPU build contracts multiply-adds (nvcc default), this engine does not
            res["max_rel_diff_vs_reference_gpu"] = float(np.nanmax(rel))
    return res


def run_batched(args, dev, stream, flush, rank):
    """The mixed 48-frame batch through mvs_batch (one graph launch per batch)."""
    import time
    import torch
    import mvs_b200 as M
    from mvs_b200 import dist, scenes
    specs = scenes.batch_workload(seed=4 + rank, n=args.batch_frames)
    rnd = scenes.GpuRenderer(dev)
    frames = []
    evals = 0
    for sp in specs:
        sc, ref_cam, cams = scenes.frame_geometry(sp.seed, sp.width, sp.height, sp.K, sp.n_src, sp.baseline,
                                                  sp.rot_deg, sp.scene)
        gray, _ = rnd.render(sc, [ref_cam] + cams)
        rel = [M.relative_pose(ref_cam.R, ref_cam.t, c.R, c.t) for c in cams]
        frames.append(dict(ref=gray[0].contiguous(), srcs=gray[1:].contiguous(), rel=rel, K1=ref_cam.K_1based,
                           depths=torch.from_numpy(scenes.inverse_depth_planes(sp.znear, sp.zfar, sp.n_planes)).to(dev),
                           window=sp.window, zfar=sp.zfar,
                           depth=torch.empty((sp.height, sp.width), device=dev),
                           labels=torch.empty((sp.height, sp.width), dtype=torch.int32, device=dev),
                           best=torch.empty((sp.height, sp.width), device=dev)))
        evals += sp.width * sp.height * sp.n_planes * sp.n_src
    t0 = time.time()
    b = M.Batch(frames, M.MOMENTS_COMPENSATED)      # autotunes on first use of this batch shape
    tune_s = time.time() - t0
    for _ in range(2):
        b.run()
    torch.cuda.synchronize()
    ms, lats = [], []
    for _ in range(max(3, args.steps)):
        flush.zero_()
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        b.run()
        c.record(stream)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(c))
        lats.append(b.latencies_ms())
    lat = np.concatenate(lats)
    batch_ms = dist.max_over_ranks(statistics.mean(ms), dev)
    # the same frames one at a time through the single-frame entry points
    seq = []
    ws_cache = {}
    for k in range(2):
        torch.cuda.synchronize()
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for f in frames:
            h, w = f["ref"].shape
            V, P = f["srcs"].shape[0], f["depths"].numel()
            desc = M.sweep_desc(w, h, V, P, f["window"], M.MOMENTS_COMPENSATED, M.SWEEP_AGGREGATED, 1e-4, 0.5,
                                f["zfar"])
            key = (w, h, V, P)
            if key not in ws_cache:
                ws_cache[key] = (torch.empty(V * P * 9, device=dev),
                                 torch.empty(M.sweep_workspace_bytes(desc) // 8 + 1, dtype=torch.int64, device=dev))
            Hb, wsb = ws_cache[key]
            M.sweep_homographies(desc, f["K1"], f["rel"], f["depths"], Hb)
            M.sweep(desc, f["ref"], f["srcs"], Hb, f["depths"], f["depth"], f["labels"], f["best"], None, wsb)
        c.record(stream)
        torch.cuda.synchronize()
        if k:
            seq.append(a.elapsed_time(c))
    kinds = {}
    for sp in specs:
        kinds[sp.kind] = kinds.get(sp.kind, 0) + 1
    ppc, ctas, order, tile_step = b.tuning
    out = {"frames": len(frames), "mix": kinds, "evals_per_batch": evals,
           "value": evals * dist.world()[1] / (batch_ms / 1e3) / 1e6, "unit": UNIT, "ms_per_batch": batch_ms,
           "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max()), "samples": int(lat.size)},
           "tuning": {"planes_per_chunk": ppc, "ctas_per_sm": ctas,
                      "order": ["frame", "largest_first", "interleaved"][order],
                      "tile": f"32 rows x (64 or 56 for windows above 9x9) - {8 * tile_step} columns",
                      "tile_step": tile_step},
           "autotune_s": tune_s, "work_items": b.work_items,
           "sequential_single_frame_ms": statistics.mean(seq), "launches_per_batch": 4,
           "planes": [sp.n_planes for sp in specs], "windows": [sp.window for sp in specs]}
    b.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["mvs", "reference"], default="mvs")
    ap.add_argument("--tgv-steps", type=int, default=3)
    ap.add_argument("--tgv-iteration", choices=("launch", "persistent"), default="launch",
                    help="TGV2 iteration form of the tgv2 leg (the on-chip persistent form for profiling)")
    ap.add_argument("--no-warm-start", dest="warm_start", action="store_false",
                    help="skip the learned TGV2 warm start")
    ap.add_argument("--warm-frames", type=int, default=8)
    ap.add_argument("--no-batch", dest="batch", action="store_false", help="skip the batched-frames workload")
    ap.add_argument("--no-reference-gpu", dest="reference_gpu", action="store_false",
                    help="skip timing the reference's own CUDA kernels on this GPU")
    ap.add_argument("--batch-frames", type=int, default=48)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fusion", dest="fusion", action="store_false")
    ap.add_argument("--no-tgv-sparse", dest="tgv_sparse", action="store_false",
                    help="skip the TGVdenoiseFromSparse timing")
    ap.add_argument("--fusion-dims", type=int, default=256, help="voxels per side of the fusion volume")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    from mvs_b200 import dist
    import mvs_b200 as M

    rank, ws, local = dist.world()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        dist.init("nccl")
    stream = torch.cuda.current_stream()

    fr, planes = make_frame(rank)
    d_ref = torch.from_numpy(fr.ref).to(dev)
    d_srcs = torch.from_numpy(np.stack(fr.srcs)).to(dev)
    d_depths = torch.from_numpy(planes).to(dev)
    desc = M.sweep_desc(W, H, V, P, WIN, M.MOMENTS_COMPENSATED, M.SWEEP_AGGREGATED, 1e-4, 0.5, 8.0)
    rel = [M.relative_pose(fr.ref_cam.R, fr.ref_cam.t, c.R, c.t) for c in fr.src_cams]
    K1 = fr.ref_cam.K_1based
    d_H = torch.empty(V * P * 9, dtype=torch.float32, device=dev)
    depth = torch.empty((H, W), dtype=torch.float32, device=dev)
    labels = torch.empty((H, W), dtype=torch.int32, device=dev)
    best = torch.empty((H, W), dtype=torch.float32, device=dev)
    cost = torch.empty((P, H, W), dtype=torch.int16, device=dev)
    wsp = torch.empty(M.sweep_workspace_bytes(desc) // 8 + 1, dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        M.sweep_homographies(desc, K1, rel, d_depths, d_H)
        M.sweep(desc, d_ref, d_srcs, d_H, d_depths, depth, None, None, cost, wsp)
        M.sweep_wta_volume(cost, d_depths, W * H, P, 8.0, depth, labels, best)

    # homography_kernel, quad_kernel (the sources' 2x2 neighbourhoods), sweep_aggregated_kernel,
    # wta_finish_kernel (the sweep's epilogue), wta_volume_kernel (WTA over the stored volume)
    launches_per_step = 5

    # clocks and throttle reasons, sampled every 20 ms from before the warm-up to the end
    clocks = ClockSampler(local).__enter__()
    clocks.wait_first()

    # --- sweep: warm-up, then K timed steps (events per step; L2 flushed between steps) ---
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    dist.barrier()
    torch.cuda.synchronize()
    t_timed0 = time.time()
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        M.sweep_homographies(desc, K1, rel, d_depths, d_H)
        kev[k][0].record(stream)
        M.sweep(desc, d_ref, d_srcs, d_H, d_depths, depth, None, None, cost, wsp)
        kev[k][1].record(stream)
        M.sweep_wta_volume(cost, d_depths, W * H, P, 8.0, depth, labels, best)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    timed_window = (t_timed0, time.time())
    dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    sweep_ms = [a.elapsed_time(b) for a, b in kev]
    total_s = dist.max_over_ranks(sum(step_ms) / 1e3, dev)
    evals = W * H * P * V
    value = evals * args.steps * ws / total_s / 1e6
    ms_per_step = total_s * 1e3 / args.steps

    # --- WTA-over-volume kernel alone (HBM-bound) ---
    torch.cuda.synchronize()
    we = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(5)]
    for a, b in we:
        flush.zero_()
        a.record(stream)
        M.sweep_wta_volume(cost, d_depths, W * H, P, 8.0, depth, labels, best)
        b.record(stream)
    torch.cuda.synchronize()
    wta_ms = statistics.median(a.elapsed_time(b) for a, b in we)

    # --- TGV2 from the WTA depth to relative energy change 1e-4 (cap 500) ---
    from mvs_b200 import hostmath as hm
    Kf = np.float32(K1)
    iK = hm.inv3_f32(Kf)
    relf = [hm.relative_f32(fr.ref_cam.R, fr.ref_cam.t, c.R, c.t) for c in fr.src_cams]
    Rs = np.stack([r[0].reshape(9) for r in relf])
    ts = np.stack([r[1] for r in relf])
    tform = M.TGV2_ITER_PERSISTENT if args.tgv_iteration == "persistent" else M.TGV2_ITER_LAUNCH
    tprm = M.tgv2_params(niters=500, warps=1, tol=1e-4, check_every=10, iteration_kernel=tform)
    u = torch.empty((H, W), dtype=torch.float32, device=dev)
    tws = torch.empty(M.tgv2_workspace_bytes(W, H, V) // 8 + 1, dtype=torch.int64, device=dev)
    wta_depth = depth.clone()
    tgv_ms, tgv_iters, tgv_e = [], 0, 0.0
    for k in range(1 + args.tgv_steps if args.tgv_steps > 0 else 0):
        u.copy_(wta_depth)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        tgv_iters, tgv_e = M.tgv2_run(d_ref, d_srcs, Kf.reshape(9), iK.reshape(9), Rs, ts, tprm, u,
                                      u_from_input=True, workspace=tws)
        b.record(stream)
        torch.cuda.synchronize()
        if k > 0:
            tgv_ms.append(a.elapsed_time(b))
    tgv_ms_frame = dist.max_over_ranks(statistics.mean(tgv_ms), dev) if tgv_ms else None

    # --- learned warm start: network prediction from (WTA depth, cost, image), then
    #     TGV2 from it with the same linearisation (WTA depth), tolerance and cap, against plain
    #     TGV2 from the WTA depth (the baseline it is measured against), averaged over held-out
    #     640x480, 8-view frames ---
    warm = None
    if tgv_ms and args.warm_start:
        from mvs_b200 import warmstart as WS
        wparams, wnorm, wmeta = WS.load_weights()
        rows = WS.evaluate(range(920000 + 100 * rank, 920000 + 100 * rank + args.warm_frames), WS.FrameConfig(),
                           wparams, wnorm, device=dev)
        pm = statistics.mean(r["plain_ms"] for r in rows)
        wm = statistics.mean(r["warm_ms"] for r in rows)
        pm, wm = dist.max_over_ranks(pm, dev), dist.max_over_ranks(wm, dev)
        er = [r["warm_energy"] / r["plain_energy"] - 1.0 for r in rows]
        reach_ms = [r["warm_ms_to_plain_energy"] for r in rows]
        rm = statistics.mean(x if x is not None else r["warm_ms"] for x, r in zip(reach_ms, rows))
        rm = dist.max_over_ranks(rm, dev)
        warm = {"frames": len(rows), "ms_per_frame_plain": pm, "ms_per_frame": wm, "speedup_vs_plain": pm / wm,
                "ms_to_plain_energy": rm, "speedup_to_plain_energy": pm / rm,
                "network_ms": statistics.mean(r["network_ms"] for r in rows),
                "prediction_energy_rel_to_plain_mean": statistics.mean(r["start_energy"] / r["plain_energy"] - 1.0
                                                                       for r in rows),
                "iterations_plain": [r["plain_iters"] for r in rows],
                "iterations_warm": [r["warm_iters"] for r in rows],
                "warm_iterations_to_plain_energy": [r["warm_iters_to_plain_energy"] for r in rows],
                "energy_rel_to_plain_mean": statistics.mean(er), "energy_rel_to_plain_max": max(er),
                "frames_with_fallback_to_plain": sum(e > 1e-4 for e in er),
                "median_abs_depth_err_m": {"plain": statistics.mean(r["plain_err"] for r in rows),
                                           "warm": statistics.mean(r["warm_err"] for r in rows)},
                "dual_start": {"sigma_pq": WS.WARM_DUAL_SIGMA, "sigma_r": WS.WARM_DUAL_SIGMA_R},
                "steps": {"warm": {"tau": WS.WARM_TAU, "sigma": WS.WARM_SIGMA},
                          "plain": {"tau": 0.02, "sigma": 1.0}},
                "network": {"weights": WS.WEIGHTS.name, "trained": wmeta},
                "includes": "network forward + TGV2 to tolerance; scenes rendered on the device, seeds held out"}

    # --- the reference's own CUDA kernels on this GPU, same frame and plane list (context for the
    #     ratios: the same evaluations, one launch per reference wrapper call) ---
    ref_gpu = None
    if args.reference_gpu and rank == 0:
        ref_gpu = run_reference_gpu(fr, planes, dev, d_ref, d_srcs, wta_depth if tgv_ms else None)

    tgv_sparse = None
    if args.tgv_sparse and rank == 0:
        tgv_sparse = run_tgv_sparse(fr, dev, d_ref, wta_depth, peaks()[0], args.reference_gpu)

    # --- batched uneven frames: 48 frames (320x240 / 640x480 rooms, 1242x375 street)
    #     with 64-256 planes, 4-8 views and 5x5-11x11 windows in one graph launch; the autotuner
    #     picks plane chunking, persistent CTAs per SM and item order ---
    batched = None
    if args.batch:
        batched = run_batched(args, dev, stream, flush, rank)

    # --- TV-L1 histogram fusion: 256^3 voxels over a 5 m cube, 40 depthmaps of
    #     640x480 with 1% depth noise and 2% outliers, 7 bins, 200 primal-dual iterations ---
    fusion = None
    if args.fusion:
        from mvs_b200 import scenes
        fi = scenes.fusion_sequence(SEED + 100 + rank, 40, W, H)
        fdims, fbins, fiters = (args.fusion_dims,) * 3, 7, 200
        nvox = fdims[0] * fdims[1] * fdims[2]
        d_maps = torch.from_numpy(np.stack(fi.depths)).to(dev)
        fK = np.stack([c.K for c in fi.cams]).astype(np.float32)
        fR = np.stack([c.R for c in fi.cams]).astype(np.float32)
        ft = np.stack([c.t for c in fi.cams]).astype(np.float32)
        vol = M.FusionVolume(fdims, fbins, fi.vol_min, fi.vol_max)
        hist_ms, tv_ms = [], []
        for k in range(2):       # first pass is the warm-up
            vol.reset()
            flush.zero_()
            a, b, c_ = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record(stream)
            vol.histogram(d_maps, fK, fR, ft, 0.05)
            b.record(stream)
            vol.tvl1(fiters, 0.1, 0.5, 1.0)
            c_.record(stream)
            torch.cuda.synchronize()
            if k:
                hist_ms.append(a.elapsed_time(b))
                tv_ms.append(b.elapsed_time(c_))
        surf = vol.extract(-1.0, 0.0, capacity=0)
        vol.close()
        hist_s = dist.max_over_ranks(hist_ms[0] / 1e3, dev)
        tv_s = dist.max_over_ranks(tv_ms[0] / 1e3, dev)
        # algorithmic HBM bytes per voxel: histogram 32 (16-byte counts in and out);
        # one iteration = U (p 12, u 4, counts 16 in; u 4, v 4 out) + P (v 4, p 12 in; p 12 out) = 68
        tv_gbs = nvox * 68 * fiters / tv_s / 1e9
        # compulsory bytes of an iteration that moves each array once (u 4, p 12, 7 uint16
        # counts 14 in; u 4, p 12 out): 46, the lower bound the two passes are held against
        tv_gbs46 = nvox * 46 * fiters / tv_s / 1e9
        fusion = {"workload": f"{args.fusion_dims}^3 voxels, 40 maps 640x480, 7 bins, 200 TV-L1 iterations",
                  "histogram_voxel_updates_per_s": nvox * 40 * ws / hist_s, "histogram_ms": hist_s * 1e3,
                  "tvl1_voxel_iterations_per_s": nvox * fiters * ws / tv_s, "tvl1_ms": tv_s * 1e3,
                  "tvl1_roofline": {"bound": "hbm", "achieved": tv_gbs, "peak": peaks()[0], "unit": "GB/s",
                                    "frac": tv_gbs / peaks()[0], "bytes_per_voxel_iteration": 68,
                                    "frac_of_compulsory_46B": tv_gbs46 / peaks()[0]}}

    if fusion is not None and rank == 0 and ws == 1 and not args.no_cpu_baseline:
        # the reference's own fusion kernels on the host cores (oracle/_ref, OpenMP over
        # blocks), on a bounded sample: a 96^3 volume of the same scene, all 40 maps, 4 iterations
        sys.path.insert(0, str(ROOT / "oracle"))
        import pyoracle as po
        if po.ref_lib() is not None:
            sdims = (96, 96, 96)
            rv = po.RefVolume(7, sdims, fi.vol_min, fi.vol_max)
            th = sum(rv.histogram(fi.depths[m], fK[m], fR[m], ft[m], 0.05) for m in range(40))
            tt = 0.0
            for _ in range(4):
                tt += rv.update_u(0.1, 0.5) + rv.update_p(1.0)
            nv = 96 ** 3
            fusion["cpu_baseline"] = {"kind": "reference", "cores": os.cpu_count(),
                                      "sample": "96^3 volume, the same 40 maps, 4 TV-L1 iterations",
                                      "histogram_voxel_updates_per_s": nv * 40 / th,
                                      "tvl1_voxel_iterations_per_s": nv * 4 / tt}

    # --- end to end through the PlaneSweep handle: host images in, host depthmap out ---
    ps = M.PlaneSweep()
    ps.setK(K1.astype(np.float32))
    ps.setPlaneDepths(planes)
    ps.setWindowSize(WIN)
    ps.setNumberofImages(V)
    ps.setZ(0.4, 8.0)
    ps.setSweepOptions(M.MOMENTS_COMPENSATED, M.SWEEP_AGGREGATED, True)
    Rsrc = np.stack([c.R for c in fr.src_cams]).astype(np.float32)
    tsrc = np.stack([c.t for c in fr.src_cams]).astype(np.float32)
    # the caller's host images: the reference and one (V, H, W) array of sources
    # in page-locked host memory, which the handle uploads from directly
    t_ref = torch.from_numpy(np.ascontiguousarray(fr.ref, dtype=np.float32)).pin_memory()
    t_srcs = torch.from_numpy(np.ascontiguousarray(np.stack(fr.srcs), dtype=np.float32)).pin_memory()
    h_ref, h_srcs = t_ref.numpy(), t_srcs.numpy()
    h_depth = np.empty((H, W), np.float32)   # the caller's depthmap, filled every frame

    def e2e_step():
        ps.set_reference(h_ref, fr.ref_cam.R, fr.ref_cam.t)
        ps.set_sources(h_srcs, Rsrc, tsrc)
        ps.RunAlgorithm()
        return ps.getDepthmap(out=h_depth)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    dist.barrier()
    # time only the e2e calls (the L2 flushes between them are excluded)
    durs = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        e2e_step()
        durs.append(time.perf_counter() - t1)
    e2e_s = dist.max_over_ranks(sum(durs), dev)
    e2e_value = evals * args.steps * ws / e2e_s / 1e6
    ps.close()

    hbm, peak_kind = peaks()
    # TGV2 iteration: 8 (8 + V) bytes of state read and written plus 4 (4 + 2V) bytes of constants
    # per pixel (u, v, p, q, r_i; T, u0, It_i, Iu_i): 208 B at V = 8
    tgv_roofline = None
    if tgv_ms:
        it_ms = tgv_ms_frame / max(tgv_iters, 1)
        tb = (8 * (8 + V) + 4 * (4 + 2 * V)) * W * H
        tgv_roofline = {"bound": "hbm", "kernel": "iteration_kernel<8> (one dependent launch per iteration)",
                        "achieved": tb / (it_ms / 1e3) / 1e9,
                        "peak": hbm, "unit": "GB/s", "frac": tb / (it_ms / 1e3) / 1e9 / hbm,
                        "bytes_per_iteration": tb, "ms_per_iteration_incl_energy_checks": it_ms,
                        "traffic": NCU_TRAFFIC["tgv2_iteration_kernel"],
                        "note": "fraction against the HBM model (208 B per pixel); the working set stays in L2 "
                                "between the back-to-back iterations. The on-chip form (MVS_TGV2_ITER_PERSISTENT) "
                                "keeps the state in shared memory: 65 MB of DRAM traffic for all 500 iterations, "
                                "14.5 us per iteration against 12.1 for this form"}
    sweep_s = statistics.median(sweep_ms) / 1e3
    # algorithmic bytes of the sweep kernel per launch: reference + 8 sources read once,
    # BF16 cost volume written once, WTA partials written once
    alg_bytes = (1 + V) * W * H * 4 + P * W * H * 2 + W * H * 8
    achieved = alg_bytes / sweep_s / 1e9
    # DRAM bytes (read + write) of one launch of each kernel in an `ncu --set full` capture of
    # this workload (one launch, L2 cold): the sweep's cost-volume writes partly stay in L2
    traffic = NCU_TRAFFIC.get("sweep_aggregated_kernel")
    wta_bytes = P * W * H * 2 + W * H * (4 + 4 + 4) + P * 4
    # FP32 roof of the sweep: SWEEP_OPS_PER_EVAL algorithmic FP32 operations per (pixel, plane,
    # view) evaluation against one FP32 operation per lane per clock
    clocks.__exit__(None, None, None)
    clock_summary = clocks.summary(timed_window)
    sm_mhz = (clock_summary or {}).get("sm_max_mhz") or 1965.0
    fp32_peak = 148 * 128 * sm_mhz * 1e6
    fp32_achieved = evals * SWEEP_OPS_PER_EVAL / sweep_s
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (bf16 cost volume)",
        "data": "synthetic: seeded ray-cast box room, 4-octave value noise (stands in for ICL-NUIM)",
        "config": {"workload": "sweep: 640x480, 8 views, 256 inverse-depth planes over [0.4, 8] m, 9x9 NCC, "
                               "compensated moments, BF16 cost volume + WTA",
                   "per_rank_frames_per_step": 1, "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": f"replicas x{ws}"},
        "roofline": {"bound": "hbm", "kernel": "sweep_aggregated_kernel", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                     "note": "the fused sweep is FP32/shared-memory issue bound; its HBM fraction is small by design",
                     "ms_per_launch": sweep_s * 1e3},
        "fp32_roofline": {"bound": "fp32 issue", "kernel": "sweep_aggregated_kernel",
                          "ops_per_eval": SWEEP_OPS_PER_EVAL, "achieved": fp32_achieved / 1e12,
                          "peak": fp32_peak / 1e12, "unit": "T FP32 ops/s", "frac": fp32_achieved / fp32_peak,
                          "peak_kind": "148 SMs x 128 FP32 lanes x max SM clock"},
        "wta_volume_roofline": {"bound": "hbm", "achieved": wta_bytes / (wta_ms / 1e3) / 1e9, "peak": hbm,
                                "unit": "GB/s", "frac": wta_bytes / (wta_ms / 1e3) / 1e9 / hbm,
                                "ms_per_launch": wta_ms, "traffic": NCU_TRAFFIC.get("wta_volume_kernel")},
        "tgv2_roofline": tgv_roofline,
        "tgv2": {"ms_per_frame_plain": tgv_ms_frame, "iterations": tgv_iters, "energy": tgv_e,
                 "tol": 1e-4, "cap": 500, "start": "WTA depth",
                 "ms_per_frame_warm_start": warm["ms_per_frame"] if warm else None, "warm_start": warm},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": (1 + V) * W * H * 4,
                "d2h_bytes_per_step": W * H * 4, "api": "mvs_ps_* PlaneSweep handle (RunAlgorithm + getDepthmap)",
                "host_inputs": "page-locked"},
        "fusion": fusion,
        "batched": batched,
        "reference_gpu": ref_gpu,
        "tgv_sparse": tgv_sparse,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clock_summary,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, secs, kind, cores, sample = cpu_reference_sample(fr, planes)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
                               "seconds": secs}
    if rank == 0:
        print(json.dumps(out), flush=True)
    dist.finish()
    return 0


if __name__ == "__main__":
    sys.exit(main())
