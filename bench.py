#!/usr/bin/env python
"""Benchmark: one space-time primal-dual iteration of the 4D reconstruction.

Workload (the 4D configuration the "s per 4D primal-dual iteration" metric is
quoted on): 10 frames of a 256^3 FP32 deforming ellipsoid phantom (30
ellipsoids displaced by u(x,t) = 4 sin(2 pi t/T + phi)(sin kx, sin ky, sin kz),
k = 2 pi/256), 36 views per frame on golden-angle low-discrepancy angles, a
512x512 detector, sid 600 mm, sdd 1000 mm, voxel-based SART (alpha 0.3),
TV weight 0.01 (Huber 0.01), temporal weight 0.1, brightness-constancy weight
0.05, the reference's ROI cut.  Synthetic, seeded data stand in for the
reference's external scans.  A step is one full primal-dual iteration over all
frames: backward warp + dual, forward warp + primal, SART over every view,
ROI mask, over-relaxation.

metric: projector GUPS over the 4D primal-dual iteration
        = frames * N^3 * views_per_frame / seconds_per_iteration / 1e9
        (each voxel-view update is one forward projection + one backprojection).

`python bench.py [--gpus N --steps K --warmup W]`; for N > 1 launch with
torch.distributed.run: each rank solves its own 10 frames (weak scaling) and
exchanges the neighbouring frames' boundary volumes with NCCL.
`--impl reference` times the reference's CPU implementation of the same step
(the reference's own projector and warp compiled from its sources, the SART and
primal-dual loop bodies restated in FP32) on the host's cores.
"""
from __future__ import annotations

import argparse
import contextlib
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
TRAFFIC_FILE = ROOT / "profiles" / "fp_corr_traffic.json"

# The single-frame workloads (the headline is the 4D iteration above).  Every
# one uses 1 mm voxels and detector pixels, sid 600 mm, sdd 1000 mm, views
# equally spaced over 360 degrees and seeded ellipsoid phantoms (centres in the
# inner 80 %, semi-axes 5-40 voxels at 256^3, scaled with the volume, additive
# densities 0.1-1).
CONFIG_SPECS = {
    1: dict(workload="plain single-frame SART, 128^3 FP32, 128 views over 360 deg, 128^2 detector, voxel-based BP, "
                     "alpha 0.3, 20 iterations, 1% Gaussian noise on the sinogram",
            n=128, det=128, views=128, ellipsoids=12, porous=False, noise=0.01, solve="sart", iters=20,
            bps=("voxel",), alpha=0.3, roi=None),
    2: dict(workload="single-frame primal-dual TV + SART, 256^3 FP32, 360 views over 360 deg, 512^2 detector, "
                     "sigma = tau = 0.2, lambda 0.01, Huber 0.01, 20 outer iterations of 1 SART sweep, "
                     "voxel- and ray-based BP",
            n=256, det=512, views=360, ellipsoids=30, porous=False, noise=0.0, solve="pd", iters=20,
            bps=("voxel", "ray"), alpha=0.3, sigma=0.2, tau=0.2, lam=0.01, huber=0.01,
            roi=(8, 8, 8, 45, 8, 8, 30, 20)),
    5: dict(workload="single-frame primal-dual TV + SART, 512^3 FP32, 720 views over 360 deg, 1024^2 detector, "
                     "100 ellipsoids on a 0.5-density porous background of random spheres (radius 2-6), "
                     "10 outer iterations, voxel- and ray-based BP",
            n=512, det=1024, views=720, ellipsoids=100, porous=True, noise=0.0, solve="pd", iters=10,
            bps=("voxel", "ray"), alpha=0.3, sigma=0.9 / 8.0, tau=1.0, lam=0.01, huber=0.01,
            roi=(16, 16, 16, 90, 16, 16, 60, 40), storages=("f32", "bf16")),
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["stt", "reference"], default="stt")
    ap.add_argument("--n", type=int, default=256, help="volume edge (voxels)")
    ap.add_argument("--frames", type=int, default=10)
    ap.add_argument("--views", type=int, default=36, help="views per frame")
    ap.add_argument("--det", type=int, default=512, help="detector edge (pixels)")
    ap.add_argument("--bp", choices=["voxel", "ray"], default="voxel")
    ap.add_argument("--no-plain", action="store_true", help="skip the per-view (plain) comparison")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-flow", action="store_true", help="skip the optical-flow leg")
    ap.add_argument("--batch-only", action="store_true",
                    help="run only the batched independent-instance solve (config 4) and print its line")
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--flow-only", action="store_true",
                    help="run only the optical-flow leg (one L1Huber_OF level at --n^3) and print its line")
    ap.add_argument("--config", type=int, choices=sorted(CONFIG_SPECS), default=None,
                    help="run only the single-frame workload of that number (1: 128^3 SART, 2: 256^3 PD TV, "
                         "5: 512^3 PD TV) and print its own line")
    ap.add_argument("--tuned", action="store_true",
                    help="with --fp-probe: autotune first, projections inside the NVTX range fp_probe")
    ap.add_argument("--tuning", default=None,
                    help="with --fp-probe --tuned or --iter-probe: launch choices (a JSON object or key=value,... "
                         "with the keys of the printed tuning: fp_variant, slab_variant, bp_variant, staged_bins, "
                         "ray_variant, staged_bins_bf16) set instead of autotuning, so that a run under ncu, whose "
                         "interception gaps fall inside the tuner's event timings, makes the choices of a plain run")
    ap.add_argument("--bp-ray-probe", action="store_true",
                    help="with --config: only run a few ray-driven backprojections at the workload's size")
    ap.add_argument("--iter-probe", action="store_true",
                    help="only the headline solver's warm-up and one iteration in an NVTX range (for ncu's launch list)")
    ap.add_argument("--persistent", action="store_true",
                    help="with --iter-probe: the persistent form (STT_SOLVE_PERSISTENT, one launch per iteration)")
    ap.add_argument("--fp64-pd-check", action="store_true",
                    help="run only the full-size FP64 check of one 4D primal-dual iteration (two frames) and print it")
    ap.add_argument("--no-configs", action="store_true",
                    help="default run: skip the single-frame workloads' sub-lines")
    ap.add_argument("--no-batch", action="store_true",
                    help="default run: skip the batched-instances leg (config 4; --batch-only runs it alone)")
    ap.add_argument("--fp-probe", action="store_true",
                    help="with --config: only project a few views with the fused forward projector "
                         "(a small command for ncu captures at that size)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
def workload(args) -> dict:
    return {"workload": f"4D primal-dual iteration, {args.frames} frames x {args.n}^3 FP32, "
                        f"{args.views} views/frame, {args.det}^2 detector",
            "frames": args.frames, "volume": [args.n] * 3, "views_per_frame": args.views,
            "detector": [args.det, args.det], "sid_mm": 600.0, "sdd_mm": 1000.0,
            "backprojector": "voxel-based" if args.bp == "voxel" else "ray-based",
            "alpha": 0.3, "tv_weight": 0.01, "huber": 0.01, "tp_weight": 0.1, "bc_weight": 0.05,
            "angles": "golden-angle low-discrepancy, consecutive across frames",
            "l2": "inputs larger than L2 (solver state ~8 GB per GPU), no flush needed"}


def pd_params(gmax: float):
    import spacetimetomography_b200 as stt

    sigma = 0.9 / 8.0  # CP_sigma = 0.9/(L*CP_tau), L = 8, CP_tau = 1 (ST_Tomography.cpp:99-102)
    lam, huber = 0.01, 0.01
    return stt.PdParams(sigma=sigma, tau=1.0, tv_w=lam, tp_w=0.1, bc_w=0.05,
                        huber_factor=1.0 / (1.0 + sigma * huber / lam), gmax=gmax)


def angles_for(args, rank: int) -> np.ndarray:
    golden = math.pi * (3.0 - math.sqrt(5.0))
    first = rank * args.frames * args.views
    return (np.arange(first, first + args.frames * args.views) * golden) % (2 * math.pi)


def build_problem(args, dev, rank: int):
    """Device state of one rank's frames plus the pinned host copy of its inputs."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    N, F, V, D = args.n, args.frames, args.views, args.det
    dims = (N, N, N)
    ang = angles_for(args, rank)
    ctx = stt.Context(dev.index or 0)
    ctx.set_geometry(dims, (1.0, 1.0, 1.0), (D, D), 1.0, 600.0, 1000.0, ang)
    params = ph.ellipsoid_params(30, dims, seed=2024, semi=(5.0 * N / 256, 40.0 * N / 256))
    T = F * max(1, int(os.environ.get("WORLD_SIZE", "1")))
    phase = 0.7
    proj = torch.empty((F, V, D, D), device=dev)
    flow = torch.empty((F, 3, N, N, N), device=dev)
    for f in range(F):
        t = rank * F + f
        truth = ph.rasterize(ph.displaced_params(params, t, T, 4.0, 2 * math.pi / N, phase), dims, dev)
        ctx.fp(truth, proj[f], view0=f * V, nviews=V)
        flow[f] = ph.deformation_flow(dims, t, t + 1, T, 4.0, 2 * math.pi / N, phase, device=dev)
    proj = ph.add_noise(proj, 0.01, seed=7 + rank)
    torch.cuda.synchronize()
    gmax = float(proj[0].max().item() / 4.0)
    st = dict(vol=torch.zeros((F + 1, N, N, N), device=dev), xbar=torch.zeros((F + 1, N, N, N), device=dev),
              xprev=torch.zeros((F, N, N, N), device=dev), ytv=torch.zeros((F, 3, N, N, N), device=dev),
              ytp=torch.zeros((F, N, N, N), device=dev), ybc=torch.zeros((F, N, N, N), device=dev),
              flow=flow, proj=proj)
    return ctx, st, gmax, ang


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms in the background."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    if PEAKS_FILE.exists():
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_launch(args):
    """DRAM bytes per k_fp_corr launch from the committed ncu capture summary, if any."""
    if TRAFFIC_FILE.exists():
        d = json.loads(TRAFFIC_FILE.read_text())
        key = f"{args.n}x{args.det}"
        if key in d:
            return d[key]
    return None


# ---------------------------------------------------------------------------
def phantom_module():
    """spacetimetomography_b200/phantom.py loaded from its file.  Importing it
    through the package would load libstt.so, which the reference arm (a CPU
    run of the reference's code) must not map."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("stt_phantom_file", ROOT / "spacetimetomography_b200" / "phantom.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


REF_SART_VIEWS = 10  # one SART call of the reference: rounds x 10 views (main.cpp:148); one round


def cpu_sample_inputs(args, threads: int) -> dict:
    """Inputs of the CPU sample (untimed): frame 0 of the phantom, its flow,
    and REF_SART_VIEWS projections of it at the reference's 36-degree steps."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bind as ob

    ph = phantom_module()
    N, D, F = args.n, args.det, args.frames
    dims = (N, N, N)
    scan = ob.Scan(N, (D, D))
    vol = ph.ellipsoid_phantom(dims, 30, seed=2024, semi=(5.0 * N / 256, 40.0 * N / 256)).numpy()
    flow = ph.deformation_flow(dims, 0, 1, F, 4.0, 2 * math.pi / N, 0.7).numpy()
    start = 13.0
    views = [ob.view_round(start, k) for k in range(REF_SART_VIEWS)]
    proj = np.stack([ob.fp32(scan, v, vol, gmode=0, threads=threads)[0] for v in views])
    return dict(ob=ob, scan=scan, vol=vol, flow=flow, start=start, views=views, proj=proj)


def cpu_reference_sample(args, threads: int, inp: dict, gpu_check=None) -> dict:
    """Times the reference's CPU implementation of one frame's share of a PD
    iteration on a bounded sample and scales it to the full iteration.  The
    sample: one SART call of the reference's ST_Tomography (10 views of
    forward projection + correction + voxel backprojection + ROI mask,
    ST_Tomography.cpp:616-808, oracle/_ref/libstt_ref_st.so), the two warps
    of one frame (warping::warp, oracle/_ref/libstt_ref.so), and one frame's
    dual and primal steps (the oracle's restatement, which is bit-identical to
    the reference's Render loop; the reference keeps those loops inside Render,
    behind its optical flow).  Without the reference build the restatement
    stands in for all of it (kind "port")."""
    ob = inp["ob"]
    N, V, F = args.n, args.views, args.frames
    dims = (N, N, N)
    vol, flow, scan = inp["vol"], inp["flow"], inp["scan"]
    use_ref = ob.REF_ST is not None and ob.REF is not None
    cut = (8, 8, 8, 45, 8, 8, 30, 20)
    if use_ref:
        out = ob.ref_st_run(scan, [[inp["start"]]], inp["proj"][None], vol[None],
                            np.zeros((1, 3) + vol.shape, np.float32), bp_mode=0, alpha=0.3, cut=cut, mode=0,
                            threads=threads, full=False)
        t_sart = out["seconds"]
        t0 = time.perf_counter()
        bw = ob.ref_warp(flow, vol, -1.0)
        ob.ref_warp(flow, vol, 1.0)
        t_warps = time.perf_counter() - t0
    else:
        raylen = np.zeros(inp["proj"].shape[1:], np.float32)
        t0 = time.perf_counter()
        ob.sart32(scan, inp["views"], np.arange(REF_SART_VIEWS), inp["proj"], 0.3, 10.0, 0, vol, raylen=raylen,
                  roi=ob.roi_mask(dims, cut), gmode=0, threads=threads)
        t_sart = time.perf_counter() - t0
        t0 = time.perf_counter()
        bw = ob.warp32(flow, vol, -1.0, threads=4)
        ob.warp32(flow, vol, 1.0, threads=4)
        t_warps = time.perf_counter() - t0
    opd = ob.OPd(0.1125, 1.0, 0.01, 0.1, 0.05, 0.9, 10.0, (ob.C.c_int * 8)(*cut))
    z = np.zeros((3,) + vol.shape, np.float32)
    t0 = time.perf_counter()
    ytv, ytp, ybc = ob.pd_dual32(dims, opd, vol, vol, bw, z, z[0], z[1])
    t_dual = time.perf_counter() - t0
    t0 = time.perf_counter()
    ob.pd_primal32(dims, opd, 0, ytp, ytp, bw, ybc, ytv, vol)
    t_primal = time.perf_counter() - t0
    sample_s = t_sart + t_warps + t_dual + t_primal
    t_iter = F * (t_warps + t_dual + t_primal + (V / REF_SART_VIEWS) * t_sart)
    gups = F * N ** 3 * V / t_iter / 1e9
    out = {"value": gups, "unit": "GUPS", "cores": threads,
           "kind": "reference" if use_ref else "port",
           "sample": (f"one frame at full size: one SART call over {REF_SART_VIEWS} views (FP + correction + voxel BP "
                      "+ ROI mask), the frame's 2 warps, dual and primal steps; scaled to "
                      f"{F} frames x {V} views.  "
                      + ("SART is the reference's ST_Tomography::SART and the warps its warping::warp (oracle/_ref, "
                         "compiled from its sources); the dual and primal steps are the oracle's restatement, "
                         "bit-identical to the reference's Render loop. " if use_ref else
                         "All restated (oracle/liboracle.so): the reference build is absent. ")
                      + f"Warp on its hard-coded 4 threads, other loops on {threads} OpenMP threads"),
           "s_per_iter": t_iter, "sample_s": sample_s,
           "per_op_s": {"sart_10_views": t_sart, "warps_2": t_warps, "dual": t_dual, "primal": t_primal}}
    if gpu_check is not None:
        out["fp64_check"] = gpu_check(ob)
    return out


def fp64_sart_check(ctx, st, args, gmax, n_views: int = 6):
    """Relative L2 of the GPU SART sweep against the FP64 oracle at full size,
    on one frame's first `n_views` views, from the current GPU state."""
    import torch

    import spacetimetomography_b200 as stt

    def run(ob):
        N, D = args.n, args.det
        scan = ob.Scan(N, (D, D))
        vol0 = st["vol"][0].detach().clone()
        order = stt.frame_order(99, 0, args.frames, 0, args.views)[:n_views]
        g = vol0.clone()
        state = torch.zeros((D, D), device=vol0.device)
        ctx.sart_sweep(g, st["proj"][0].contiguous(), order, 0.3, gmax, 0, state, view_offset=0,
                       roi_cut=(8, 8, 8, 45, 8, 8, 30, 20))
        torch.cuda.synchronize()
        ang = angles_for(args, 0)
        views = [ob.view_angle(a) for a in ang[:args.views]]
        roi = ob.roi_mask(scan.dims, (8, 8, 8, 45, 8, 8, 30, 20)).astype(np.float64)
        ref, _ = ob.sart64(scan, views, order, st["proj"][0].cpu().numpy().astype(np.float64), 0.3, gmax, 0,
                           vol0.cpu().numpy().astype(np.float64), roi=roi, threads=os.cpu_count() or 1)
        return {"sart_rel_l2_vs_fp64": ob.rel_l2(g.cpu().numpy(), ref),
                "sample": f"SART over {n_views} views of frame 0 at {N}^3/{D}^2 from the solver's current state"}

    return run


def fp64_pd_iteration_check(args, dev, stream, ob) -> dict:
    """One whole 4D primal-dual iteration at the workload's full size against
    the FP64 oracle, per state: two frames of the sequence (frame 0 takes the
    first-frame primal, frame 1 the forward warp of frame 0's Y_bc), every
    view of each frame (36 at the default size), from a state one GPU
    iteration into the solve (non-zero duals).  The GPU's graph-captured
    solver and the oracle's reference-ordered loop (backward warp, dual,
    forward warp, primal, SART with voxel BP, ROI mask, over-relaxation) start
    from the same FP32 state; the sticky ray lengths start at zero in both."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    N, V, D, F = args.n, args.views, args.det, 2
    dims = (N, N, N)
    ang = angles_for(args, 0)[:F * V]
    ctx = stt.Context(dev.index or 0)
    ctx.set_geometry(dims, (1.0, 1.0, 1.0), (D, D), 1.0, 600.0, 1000.0, ang)
    params = ph.ellipsoid_params(30, dims, seed=2024, semi=(5.0 * N / 256, 40.0 * N / 256))
    proj = torch.empty((F, V, D, D), device=dev)
    flow = torch.empty((F, 3, N, N, N), device=dev)
    vol = torch.empty((F + 1, N, N, N), device=dev)
    for f in range(F):
        truth = ph.rasterize(ph.displaced_params(params, f, args.frames, 4.0, 2 * math.pi / N, 0.7), dims, dev)
        ctx.fp(truth, proj[f], view0=f * V, nviews=V)
        flow[f] = ph.deformation_flow(dims, f, f + 1, args.frames, 4.0, 2 * math.pi / N, 0.7, device=dev)
        vol[f] = truth * 0.8
    vol[F] = vol[F - 1]
    torch.cuda.synchronize()
    gmax = float(proj[0].max().item() / 4.0)
    pd = pd_params(gmax)
    z = lambda *s_: torch.zeros(s_, device=dev)  # noqa: E731
    st = dict(vol=vol, xbar=vol.clone(), xprev=z(F, N, N, N), ytv=z(F, 3, N, N, N), ytp=z(F, N, N, N),
              ybc=z(F, N, N, N), flow=flow, proj=proj)
    s1 = stt.Solver(ctx, st, F, V, pd, alpha=0.3, bp_mode=0, seed=5, mode=stt.SOLVE_GRAPH)
    s1.iterate(1, stream)  # into the solve: non-zero duals
    torch.cuda.synchronize()
    s1.close()
    start = {k: v.detach().cpu().numpy().copy() for k, v in st.items()}
    s2 = stt.Solver(ctx, st, F, V, pd, alpha=0.3, bp_mode=0, seed=11, mode=stt.SOLVE_GRAPH)
    s2.iterate(1, stream)
    torch.cuda.synchronize()
    s2.poll_status(stream)
    s2.close()
    gpu = {k: v.detach().cpu().numpy() for k, v in st.items()}
    ctx.close()
    del st, proj, flow, vol
    torch.cuda.empty_cache()
    pp = [pd.sigma, pd.tau, pd.tv_w, pd.tp_w, pd.bc_w, pd.huber_factor, gmax]
    scan = ob.Scan(N, (D, D))
    orders = [stt.frame_order(11, 0, F, f, V) for f in range(F)]
    raylen = [np.zeros((D, D), np.float64) for _ in range(F)]
    t0 = time.perf_counter()
    from spacetimetomography_b200.api import REFERENCE_CUT

    ref = ob.pd_iteration(scan, ang, start, F, V, pp, tuple(pd.cut), REFERENCE_CUT, 0.3, 0, orders, raylen,
                          fp64=True)
    t_ref = time.perf_counter() - t0
    out = {k: [ob.rel_l2(gpu[k][f], ref[k][f]) for f in range(F)]
           for k in ("vol", "xbar", "xprev", "ytv", "ytp", "ybc")}
    out["sample"] = (f"one PD iteration of frames 0-1 at {N}^3/{D}^2, {V} views each, from one GPU iteration into "
                     "the solve; per state, per frame: relative L2 of the GPU (FP32) against the FP64 oracle")
    out["oracle_s"] = t_ref
    return out


# ---------------------------------------------------------------------------
@contextlib.contextmanager
def c_stdout_to_stderr():
    """The reference's C++ code prints progress with std::cout; keep it off
    stdout, which carries only the JSON line."""
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        yield
    finally:
        try:
            ctypes.CDLL(None).fflush(None)
        except OSError:
            pass
        os.dup2(saved, 1)
        os.close(saved)


FLOW_BYTES_PER_VOXEL = 152  # minimal state per flow iteration: v 3, y 10, v-extrapolation 3 r/w, grad/ut 4 read


def flow_bench(args, dev, stream, rank: int) -> dict:
    """One level of optical_flow::L1Huber_OF at N^3 between two phantom frames:
    per-iteration device time (primal + dual over the whole volume), from two
    solves that differ only in their iteration count."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    N = args.n
    dims = (N, N, N)
    params = ph.ellipsoid_params(30, dims, seed=2024, semi=(5.0 * N / 256, 40.0 * N / 256))
    T = args.frames
    i1 = ph.rasterize(ph.displaced_params(params, 0, T, 4.0, 2 * math.pi / N, 0.7), dims, dev)
    i2 = ph.rasterize(ph.displaced_params(params, 1, T, 4.0, 2 * math.pi / N, 0.7), dims, dev)
    V = torch.zeros((3,) + dims, device=dev)
    Y = torch.zeros((10,) + dims, device=dev)
    cut = (8, 8, 8, 45, 8, 8)
    roi = tuple(int(c * (N / 256.0)) for c in cut)
    iters = 200

    def run(max_iter):
        f = stt.Flow(dims, stt.FlowParams(tol=0.0, max_iter=max_iter, n_warps=1, scales=1, cut=cut), device=dev.index or 0)
        V.zero_()
        Y.zero_()
        torch.cuda.synchronize()
        f.level(i1, i2, V, Y, roi, stream=stream)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        f.level(i1, i2, V, Y, roi, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        its, _ = f.stats()
        f.close()
        return e0.elapsed_time(e1) / 1000.0, int(its[0])

    t_long, n_long = run(iters - 1)
    t_short, n_short = run(0)
    t_it = (t_long - t_short) / (n_long - n_short)
    peak, peak_kind = peaks()
    achieved = FLOW_BYTES_PER_VOXEL * N ** 3 / t_it / 1e9
    out = {"workload": f"L1Huber_OF level, {N}^3, ROI cut {cut}, {iters} iterations, 1 warp",
           "ms_per_iteration": 1000.0 * t_it, "gvoxel_iter_per_s": N ** 3 / t_it / 1e9,
           "roofline": {"bound": "hbm", "kernel": "k_flow_primal + k_flow_dual", "achieved": achieved,
                        "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                        "algorithmic_bytes_per_voxel": FLOW_BYTES_PER_VOXEL,
                        "moved_bytes_per_voxel": 212,
                        "note": "moved per iteration: primal reads y 10, u 3, tau 3, v 3 and writes v 3 (ROI); "
                                "dual reads v 3, v_old 3, u 4, sigma2 1, y 10 and writes y 10"}}
    # the whole multiscale solve between the same frames with the reference's
    # parameters (tol 0.1, 3000 iterations, 3 warps, 3 scales, the ROI cut):
    # the warps stop on their residuals
    fm = stt.Flow(dims, stt.FlowParams(cut=cut), device=dev.index or 0)
    ms = []
    for _ in range(2):  # (the first is a warm-up)
        V.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fm.multiscale(i1, i2, V, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    its, _ = fm.stats()
    fm.close()
    out["multiscale"] = {"s": ms[-1] / 1000.0, "iterations_per_level_and_warp": its.tolist(),
                         "workload": f"L1Huber_OF_MultiScale3D, {N}^3, tol 0.1, lambda 1.2, Huber 1, 3000 "
                                     "iterations, 3 warps, 3 scales (eta 0.65), ROI cut, zero start"}
    if rank == 0 and not args.no_cpu:
        out["cpu_baseline"] = flow_cpu_sample(i1, i2)
    return out


def flow_cpu_sample(i1, i2) -> dict:
    """Per-iteration time of L1Huber_OF on the host cores: the reference's own
    optical_flow.h (oracle/_ref, OpenMP on every core) when it was built, else
    the one-thread oracle restatement; two runs that differ only in their
    iteration count, on the 128^3 corner of the bench images."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bind as ob

    n, k = 128, 31
    sl = (slice(0, n),) * 3
    a, b = i1[sl].contiguous().cpu().numpy(), i2[sl].contiguous().cpu().numpy()
    z3, z10 = np.zeros((3, n, n, n), np.float32), np.zeros((10, n, n, n), np.float32)
    cores = os.cpu_count() or 1
    use_ref = ob.REF is not None

    def run(max_iter):
        t0 = time.perf_counter()
        with c_stdout_to_stderr():
            if use_ref:
                ob.ref_flow_level(a, b, z3, z10, (0,) * 6, tol=0.0, max_iter=max_iter, n_warps=1, threads=cores)
            else:
                ob.flow_level32(a, b, z3, z10, (0,) * 6, tol=0.0, max_iter=max_iter, n_warps=1)
        return time.perf_counter() - t0

    t_it = (run(k - 1) - run(0)) / (k - 1)
    return {"value": n ** 3 / t_it / 1e9, "unit": "Gvoxel-iterations/s", "cores": cores if use_ref else 1,
            "kind": "reference" if use_ref else "port",
            "sample": f"optical_flow::L1Huber_OF one level, {n}^3, {k} minus 1 iterations, no ROI"
                      + (" (the reference's code, OpenMP)" if use_ref else " (oracle port, one thread)")}


# ---------------------------------------------------------------------------
# Single-frame workloads (CONFIG_SPECS)

def config_problem(cid: int, dev):
    """The workload's context (geometry), phantom and sinogram on the device;
    G_Max = max(sinogram)/4 as SetData forms it (ST_Tomography.cpp:356-357)."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    c = CONFIG_SPECS[cid]
    N, D, V = c["n"], c["det"], c["views"]
    dims = (N, N, N)
    ang = ph.equispaced_views(V)
    ctx = stt.Context(dev.index or 0)
    ctx.set_geometry(dims, (1.0, 1.0, 1.0), (D, D), 1.0, 600.0, 1000.0, ang)
    s = N / 256.0
    bg = ph.porous_background(dims, 77, N ** 3 // 1000, device=dev) if c["porous"] else None
    truth = ph.rasterize(ph.ellipsoid_params(c["ellipsoids"], dims, seed=100 + cid, semi=(5.0 * s, 40.0 * s)), dims,
                         dev, background=bg)
    proj = torch.empty((V, D, D), device=dev)
    ctx.fp(truth, proj)
    if c["noise"] > 0:
        proj = ph.add_noise(proj, c["noise"], seed=cid)
    torch.cuda.synchronize()
    return ctx, truth, proj.contiguous(), float(proj.max().item()) / 4.0


def _timed(stream, fn, reps: int) -> float:
    """Seconds per call of fn() over `reps` calls, CUDA events on `stream`."""
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1000.0 / max(reps, 1)


def gather_ceilings(ctx, vol, views, D, dev, stream) -> dict:
    """The gather ceiling (stt_gather_ceiling) over `views`, in both corner
    fetches: eight loads per sample, and two tld4 texture gathers (where the
    textures bind).  Samples per view and Gsamples/s of each, and which fetch
    the tuned projector uses."""
    import torch

    gimg = torch.empty((D, D), device=dev)
    gcount = torch.zeros((D, D), dtype=torch.int32, device=dev)
    out = {}
    forms = [("loads", False)] + ([("tld4", True)] if ctx.fp_texture_ok(vol) else [])
    for name, tex in forms:
        gsamples = 0
        for v in views:
            ctx.gather_ceiling(vol, v, gimg, gcount, stream=stream, texture=tex)
            torch.cuda.synchronize()
            gsamples += int(gcount.sum().item())
        it = iter(list(views) * 2)
        t = _timed(stream, lambda: (lambda v: ctx.gather_ceiling(vol, v, gimg, stream=stream, texture=tex))(next(it)),
                   len(views))
        out[name] = {"gsamples_per_s": gsamples / len(views) / t / 1e9, "s_per_view": t,
                     "samples_per_view": gsamples / len(views)}
    out["projector_fetch"] = "tld4" if ctx.get_tuning()["fp_variant"] in (10, 11) and "tld4" in out else "loads"
    return out


def _pd_state(N, proj, dev, storage="f32"):
    """A one-frame solver state; storage "bf16": the primal volumes and the
    sinogram in torch.bfloat16 (stt_solve_cfg.storage)."""
    import torch

    z = lambda *s: torch.zeros(s, device=dev)  # noqa: E731
    zp = lambda *s: torch.zeros(s, device=dev, dtype=torch.bfloat16 if storage == "bf16" else torch.float32)  # noqa
    p = proj[None] if storage == "f32" else proj[None].to(torch.bfloat16)
    return dict(vol=zp(2, N, N, N), xbar=zp(2, N, N, N), xprev=zp(1, N, N, N), ytv=z(1, 3, N, N, N),
                ytp=z(1, N, N, N), ybc=z(1, N, N, N), flow=z(1, 3, N, N, N), proj=p)


def config_solve(cid, ctx, proj, truth, gmax, bp, dev, stream, iters: int, reps: int, storage="f32",
                 keep=False) -> dict:
    """One solve of the workload; times `reps` of its iterations after one
    warm-up iteration and reports the error to the phantom after `iters`.
    storage "bf16": the primal volumes and the sinogram stored in BF16.  keep:
    the result volume (FP32) is returned under "_result"."""
    import torch

    import spacetimetomography_b200 as stt

    c = CONFIG_SPECS[cid]
    N, V = c["n"], c["views"]
    bp_mode = 0 if bp == "voxel" else 1
    if c["solve"] == "sart":
        vol = torch.zeros((N, N, N), device=dev)
        state = torch.zeros(proj.shape[1:], device=dev)
        it = [0]

        def one():
            ctx.sart_sweep(vol, proj, stt.permutation(1000 * cid + it[0], V), c["alpha"], gmax, bp_mode, state,
                           stream=stream)
            it[0] += 1
        one()
        t = _timed(stream, one, reps)
        for _ in range(max(0, iters - 1 - reps)):
            one()
        launches = None
        result = vol
    else:
        st = _pd_state(N, proj, dev, storage)
        sg, lam = c["sigma"], c["lam"]
        pd = stt.PdParams(sigma=sg, tau=c["tau"], tv_w=lam, tp_w=0.0, bc_w=0.0,
                          huber_factor=1.0 / (1.0 + sg * c["huber"] / lam), gmax=gmax, cut=c["roi"])
        solver = stt.Solver(ctx, st, 1, V, pd, alpha=c["alpha"], bp_mode=bp_mode, roi_cut=c["roi"], seed=cid,
                            mode=stt.SOLVE_GRAPH, storage=storage)

        def one():
            solver.iterate(1, stream)
        one()
        t = _timed(stream, one, reps)
        for _ in range(max(0, iters - 1 - reps)):
            one()
        torch.cuda.synchronize()
        solver.poll_status(stream)
        launches = solver.stats()[0]
        result = st["vol"][0].float()
    torch.cuda.synchronize()
    err = float((result - truth).norm() / truth.norm())
    out = {"s_per_iter": t, "gups": N ** 3 * V / t / 1e9, "iterations_run": max(iters, 1 + reps),
           "rel_l2_to_phantom": err, "launches_per_iter": launches, "storage": storage}
    if keep:
        out["_result"] = result.clone()
    if c["solve"] != "sart":
        solver.close()
    return out


def fp_bp_split(ctx, c, vol, proj, gmax, dev, stream) -> dict:
    """Per-view times of the fused forward projector (stt_fp_correction, which
    also writes the z-fastest copy for x-dominant views) and of the two
    backprojectors through the per-view ABI, the samples per view (the
    reference's sample counts, stt_fp's weight output) and the FP roofline."""
    import torch

    N, D, V = c["n"], c["det"], c["views"]
    nv = min(V, 32)
    views = [int(v) for v in np.linspace(0, V - 1, nv)]
    corr = torch.empty((D, D), device=dev)
    rl = torch.zeros((D, D), device=dev)
    for v in views[:3]:
        ctx.fp_correction(vol, proj[v], rl, corr, v, stream=stream)
    it = iter(views * 2)
    t_fp = _timed(stream, lambda: (lambda v: ctx.fp_correction(vol, proj[v], rl, corr, v, stream=stream))(next(it)), nv)
    scratch = vol.clone()
    it = iter(views * 2)
    t_bpv = _timed(stream, lambda: (lambda v: ctx.bp_voxel(corr, scratch, 0.3, gmax, v, stream=stream))(next(it)), nv)
    it = iter(views * 2)
    t_bpr = _timed(stream, lambda: (lambda v: ctx.bp_ray(corr, scratch, gmax, v, stream=stream))(next(it)), nv)
    w = torch.zeros((4, D, D), device=dev)
    img = torch.zeros((4, D, D), device=dev)
    samples = 0.0
    for k, v in enumerate(views[::max(1, nv // 4)][:4]):
        ctx.fp(vol, img[k:k + 1], view0=v, nviews=1, weight=w[k:k + 1], stream=stream)
    torch.cuda.synchronize()
    samples = float(w.sum().item()) / 4
    # the gather ceiling over the same views: the projector's gathers and
    # interpolation alone (stt_gather_ceiling), its own samples counted, in
    # the corner fetch the tuned projector uses
    gc = gather_ceilings(ctx, vol, views, D, dev, stream)
    ceiling = gc[gc["projector_fetch"]]["gsamples_per_s"]
    ctx.poll_status(stream)
    del scratch
    peak, peak_kind = peaks()
    fp_bytes = 4 * N ** 3 + 12 * D * D
    key = f"{N}x{D}"
    traffic = None
    if TRAFFIC_FILE.exists():
        traffic = json.loads(TRAFFIC_FILE.read_text()).get(key)
    return {"views_timed": nv, "fp_s_per_view": t_fp, "bp_voxel_s_per_view": t_bpv, "bp_ray_s_per_view": t_bpr,
            "fp_gups": N ** 3 / t_fp / 1e9, "bp_voxel_gups": N ** 3 / t_bpv / 1e9, "bp_ray_gups": N ** 3 / t_bpr / 1e9,
            "samples_per_view": samples, "fp_gsamples_per_s": samples / t_fp / 1e9,
            "gather_ceiling": {**gc, "fp_frac": samples / t_fp / 1e9 / ceiling,
                               "kernel": "k_gather_ceiling (stt_gather_ceiling): the projector's cell, its 8 corners "
                                         "(8 loads, or 2 tld4 gathers) and trilinear interpolation per sample, packed "
                                         "pairs, no march control; fp_frac against the projector's own fetch"},
            "roofline": {"bound": "hbm", "kernel": "k_fp_corr / k_fp_corr_slab (forward projection + correction)",
                         "achieved": fp_bytes / t_fp / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": fp_bytes / t_fp / 1e9 / peak, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": fp_bytes, "traffic": traffic,
                         "note": ("volume L2-resident (%.0f MiB < 126 MB L2)" % (4 * N ** 3 / 2 ** 20))
                         if 4 * N ** 3 < 126e6 else "volume larger than L2: streamed from HBM every view"}}


def config_e2e(cid, ctx, proj, gmax, dev, stream) -> dict:
    """One step end to end: the step's inputs (sinogram, start volume) from
    pinned host memory to the device, one iteration (voxel-based BP), the
    volume back to pinned host memory; all inside the timed region."""
    import torch

    import spacetimetomography_b200 as stt

    c = CONFIG_SPECS[cid]
    N, V = c["n"], c["views"]
    hproj = proj.detach().cpu().pin_memory()
    hvol = torch.zeros((N, N, N)).pin_memory()
    hout = torch.empty((N, N, N)).pin_memory()
    if c["solve"] == "sart":
        vol = torch.empty((N, N, N), device=dev)
        state = torch.zeros(proj.shape[1:], device=dev)
        dproj = torch.empty_like(proj)

        def step():
            with torch.cuda.stream(stream):
                dproj.copy_(hproj, non_blocking=True)
                vol.copy_(hvol, non_blocking=True)
                state.zero_()
            ctx.sart_sweep(vol, dproj, stt.permutation(7, V), c["alpha"], gmax, 0, state, stream=stream)
            with torch.cuda.stream(stream):
                hout.copy_(vol, non_blocking=True)
        step()
        t = _timed(stream, step, 2)
    else:
        dproj = torch.empty_like(proj)
        st = _pd_state(N, dproj, dev)
        sg, lam = c["sigma"], c["lam"]
        pd = stt.PdParams(sigma=sg, tau=c["tau"], tv_w=lam, tp_w=0.0, bc_w=0.0,
                          huber_factor=1.0 / (1.0 + sg * c["huber"] / lam), gmax=gmax, cut=c["roi"])
        solver = stt.Solver(ctx, st, 1, V, pd, alpha=c["alpha"], bp_mode=0, roi_cut=c["roi"], seed=cid,
                            mode=stt.SOLVE_GRAPH)

        def step():
            with torch.cuda.stream(stream):
                dproj.copy_(hproj, non_blocking=True)
                st["vol"][0].copy_(hvol, non_blocking=True)
                st["vol"][1].copy_(st["vol"][0])
                st["xbar"].copy_(st["vol"])
                for k in ("xprev", "ytv", "ytp", "ybc"):
                    st[k].zero_()
            solver.iterate(1, stream)
            with torch.cuda.stream(stream):
                hout.copy_(st["vol"][0], non_blocking=True)
        step()
        t = _timed(stream, step, 2)
        solver.close()
    return {"value": N ** 3 * V / t / 1e9, "unit": "GUPS", "h2d_bytes_per_step": hproj.numel() * 4 + hvol.numel() * 4,
            "d2h_bytes_per_step": hout.numel() * 4, "s_per_step": t,
            "through": "pinned host copies on the solve's stream around stt_sart_sweep / stt_solver_iterate, in line "
                       "(no overlap of one step's copies with another's compute)"}


def config_fp64_check(cid, ctx, truth, proj, gmax, dev, stream) -> dict:
    """Error of the CUDA path against the FP64 oracle on a bounded sample at
    the workload's full size: one SART sweep over a few views from the
    phantom scaled by 0.8 (configs 1 and 2); at 512^3 (whose FP64 projection
    of a 1024^2 view takes minutes on the host) the forward projection of a
    64-row band of one view and the voxel backprojection of one view's
    correction."""
    import torch

    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bind as ob

    c = CONFIG_SPECS[cid]
    N, D, V = c["n"], c["det"], c["views"]
    scan = ob.Scan(N, (D, D))
    ang = np.arange(V) * (2 * math.pi / V)
    threads = os.cpu_count() or 1
    if N <= 256:
        nv = 8 if N <= 128 else 3
        order = [int(v) for v in np.linspace(0, V - 1, nv)]
        v0 = (truth * 0.8).contiguous()
        g = v0.clone()
        state = torch.zeros((D, D), device=dev)
        ctx.sart_sweep(g, proj, order, c["alpha"], gmax, 0, state, stream=stream)
        torch.cuda.synchronize()
        views = [ob.view_angle(a) for a in ang]
        ref, _ = ob.sart64(scan, views, order, proj.cpu().numpy().astype(np.float64), c["alpha"], gmax, 0,
                           v0.cpu().numpy().astype(np.float64), threads=threads)
        return {"sart_rel_l2_vs_fp64": ob.rel_l2(g.cpu().numpy(), ref),
                "sample": f"one SART sweep over {nv} of the {V} views from 0.8 x phantom, voxel-based BP"}
    rows = slice(D // 2 - 32, D // 2 + 32)
    v = V // 8  # an oblique view (45 degrees)
    img = torch.zeros((1, D, D), device=dev)
    ctx.fp(truth, img, view0=v, nviews=1, stream=stream)
    torch.cuda.synchronize()
    ref_band = ob.fp64_rows(scan, ob.view_angle(ang[v]), truth.cpu().numpy().astype(np.float64), rows.start,
                            rows.stop - rows.start, threads=threads)
    fp_err = ob.rel_l2(img[0, rows].cpu().numpy(), ref_band)
    corr = torch.zeros((D, D), device=dev)
    rl = torch.zeros((D, D), device=dev)
    ctx.fp_correction((truth * 0.8).contiguous(), proj[v], rl, corr, v, stream=stream)
    vol = (truth * 0.8).contiguous()
    ctx.bp_voxel(corr, vol, c["alpha"], gmax, v, stream=stream)
    torch.cuda.synchronize()
    base = (truth * 0.8).cpu().numpy().astype(np.float64)
    ref_vol = ob.bp_voxel64(scan, ob.view_angle(ang[v]), corr.cpu().numpy().astype(np.float64), c["alpha"], gmax,
                            base.copy())
    upd = vol.cpu().numpy().astype(np.float64) - base
    bp_err = ob.rel_l2(upd, ref_vol - base)
    return {"fp_band_rel_l2_vs_fp64": fp_err, "bp_voxel_update_rel_l2_vs_fp64": bp_err,
            "sample": f"view {v} (45 deg): forward projection of detector rows {rows.start}-{rows.stop - 1}, and the "
                      "voxel backprojection of its correction (the update it adds to 0.8 x phantom)"}


def config_cpu_baseline(cid, args) -> dict:
    """The reference's own SART call (10 views of FP + correction + voxel BP +
    ROI mask, oracle/_ref) timed on the host cores at a bounded size, scaled to
    one iteration of the workload: at 128^3 and 256^3 at the workload's own
    size; at 512^3 / 1024^2 at 256^3 / 512^2, scaled by 8 (the per-view work
    of both the projector, W*H rays of N/sd samples, and the voxel
    backprojection, N^3 voxels, grows 8-fold)."""
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bind as ob

    c = CONFIG_SPECS[cid]
    if ob.REF_ST is None:
        return None
    ph = phantom_module()
    N, D = (c["n"], c["det"]) if c["n"] <= 256 else (256, 512)
    scale = 1.0 if c["n"] <= 256 else 8.0
    threads = os.cpu_count() or 1
    dims = (N, N, N)
    vol = ph.ellipsoid_phantom(dims, c["ellipsoids"], seed=100 + cid, semi=(5.0 * N / 256, 40.0 * N / 256)).numpy()
    scan = ob.Scan(N, (D, D))
    views = [ob.view_round(13.0, k) for k in range(REF_SART_VIEWS)]
    proj = np.stack([ob.fp32(scan, v, vol, gmode=0, threads=threads)[0] for v in views])
    with c_stdout_to_stderr():
        out = ob.ref_st_run(scan, [[13.0]], proj[None], vol[None], np.zeros((1, 3) + vol.shape, np.float32),
                            bp_mode=0, alpha=c["alpha"], cut=(8, 8, 8, 45, 8, 8, 30, 20), mode=0, threads=threads,
                            full=False)
    t_iter = out["seconds"] * scale * c["views"] / REF_SART_VIEWS
    return {"value": c["n"] ** 3 * c["views"] / t_iter / 1e9, "unit": "GUPS", "cores": threads, "kind": "reference",
            "sample": f"the reference's ST_Tomography::SART over {REF_SART_VIEWS} views at {N}^3 / {D}^2 "
                      f"(oracle/_ref), {threads} OpenMP threads, scaled to {c['views']} views"
                      + (" and by 8 to 512^3 / 1024^2" if scale != 1.0 else "")
                      + ("; the primal-dual steps (under 1 % of the iteration on the host) are not in the sample"
                         if c["solve"] == "pd" else ""),
            "s_per_iter": t_iter}


def config_bench(cid, args, dev, stream, rank=0, full=False) -> dict:
    """The line of one single-frame workload (see CONFIG_SPECS).  full: run
    the whole configured solve per variant; otherwise a warm-up and two timed
    iterations (as the default run's sub-line)."""
    import torch

    c = CONFIG_SPECS[cid]
    N, D, V = c["n"], c["det"], c["views"]
    ctx, truth, proj, gmax = config_problem(cid, dev)
    out = {"config": {"workload": c["workload"], "volume": [N] * 3, "detector": [D, D], "views": V,
                      "iterations": c["iters"], "data": "synthetic (seeded phantom)"},
           "metric": "projector GUPS over one iteration", "unit": "GUPS", "dtype": "f32", "variants": {}}
    reps = 3 if N <= 256 else 2
    out["tuning"] = ctx.autotune(stream)  # the launch choices for this geometry (untimed)
    storages = c.get("storages", ("f32",))
    for bp in c["bps"]:
        res = {}
        for sto in storages:
            v = config_solve(cid, ctx, proj, truth, gmax, bp, dev, stream, c["iters"] if full else 1 + reps, reps,
                             storage=sto, keep=len(storages) > 1)
            res[sto] = v.pop("_result", None)
            out["variants"][f"{sto}_{bp}"] = v
            torch.cuda.empty_cache()
        if "bf16" in res and "f32" in res:
            # BF16 storage against FP32 storage after the same iterations (the
            # FP32 solve's own error against FP64 is the fp64_check leg's)
            a, b = res["bf16"], res["f32"]
            out["variants"][f"bf16_{bp}"]["rel_l2_to_f32_storage"] = float((a - b).norm() / b.norm())
        del res
        torch.cuda.empty_cache()
    out["value"] = out["variants"]["f32_voxel"]["gups"]
    out["ms_per_step"] = 1000.0 * out["variants"]["f32_voxel"]["s_per_iter"]
    split = fp_bp_split(ctx, c, (truth * 0.8).contiguous(), proj, gmax, dev, stream)
    out["roofline"] = split.pop("roofline")
    out["fp_bp"] = split
    out["e2e"] = config_e2e(cid, ctx, proj, gmax, dev, stream)
    if rank == 0 and not args.no_cpu:
        out["fp64_check"] = config_fp64_check(cid, ctx, truth, proj, gmax, dev, stream)
        out["cpu_baseline"] = config_cpu_baseline(cid, args)
    ctx.close()
    del truth, proj
    torch.cuda.empty_cache()
    return out


_TUNING_KEYS = ("fp_variant", "slab_variant", "bp_variant", "staged_bins", "ray_variant", "staged_bins_bf16")


def tune_or_set(ctx, stream, tuning_json) -> dict:
    """Autotunes the context, or sets the choices a JSON object names."""
    if tuning_json is None:
        return ctx.autotune(stream)
    if tuning_json.lstrip().startswith("{"):
        t = json.loads(tuning_json)
    else:  # key=value,key=value
        t = dict(kv.split("=", 1) for kv in tuning_json.split(",") if kv)
    unknown = set(t) - set(_TUNING_KEYS)
    if unknown:
        raise SystemExit(f"--tuning: unknown keys {sorted(unknown)}")
    ctx.set_tuning(**{k: int(t[k]) for k in _TUNING_KEYS if k in t})
    return ctx.get_tuning()


def fp_probe(cid, dev, stream, tuned=False, tuning=None) -> None:
    """A few fused forward projections at the workload's size and nothing else
    (the command ncu captures for the roofline's traffic at that size).  With
    `tuned` the context is autotuned first (or given the choices `tuning`
    names) and the projections run inside the NVTX range "fp_probe" (so that a
    capture can skip the tuner's launches)."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    c = CONFIG_SPECS[cid]
    N, D, V = c["n"], c["det"], c["views"]
    ctx = stt.Context(dev.index or 0)
    ctx.set_geometry((N, N, N), (1.0, 1.0, 1.0), (D, D), 1.0, 600.0, 1000.0, ph.equispaced_views(V))
    vol = ph.rasterize(ph.ellipsoid_params(c["ellipsoids"], (N, N, N), seed=100 + cid,
                                           semi=(5.0 * N / 256, 40.0 * N / 256)), (N, N, N), dev)
    b = torch.zeros((D, D), device=dev)
    rl = torch.zeros((D, D), device=dev)
    corr = torch.zeros((D, D), device=dev)
    if tuned:
        print(json.dumps({"tuning": tune_or_set(ctx, stream, tuning)}), flush=True)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("fp_probe")
    for v in (0, V // 8, V // 4, 3 * V // 8):  # about 0, 45, 90, 135 degrees (0, 40, 90, 130 for 36 views)
        ctx.fp_correction(vol, b, rl, corr, v, stream=stream)
    torch.cuda.synchronize()
    if tuned:
        torch.cuda.nvtx.range_pop()
    ctx.poll_status(stream)
    ctx.close()


def bp_ray_probe(cid, dev, stream) -> None:
    """A few ray-driven backprojections at the workload's size, each view with
    both scatters (global atomics, then the shared-memory slab box) and the
    normalising update, and nothing else (the command ncu captures for the
    scatters' profile)."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    c = CONFIG_SPECS[cid]
    N, D, V = c["n"], c["det"], c["views"]
    ctx = stt.Context(dev.index or 0)
    ctx.set_geometry((N, N, N), (1.0, 1.0, 1.0), (D, D), 1.0, 600.0, 1000.0, ph.equispaced_views(V))
    vol = torch.zeros((N, N, N), device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    corr = torch.rand((D, D), device=dev, generator=g) - 0.5
    for v in (0, V // 8, V // 4, 3 * V // 8):  # about 0, 45, 90, 135 degrees (0, 40, 90, 130 for 36 views)
        for rv in (0, 1):  # both scatters: global vector atomics, the shared-memory slab box
            ctx.set_tuning(ray_variant=rv)
            ctx.bp_ray(corr, vol, 1e9, v, stream=stream)
    torch.cuda.synchronize()
    ctx.close()


def run_config_only(args) -> int:
    import torch

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    if args.fp_probe:
        fp_probe(args.config, dev, stream, tuned=args.tuned, tuning=args.tuning)
        return 0
    if args.bp_ray_probe:
        bp_ray_probe(args.config, dev, stream)
        return 0
    clocks = ClockSampler(0)
    clocks.start()
    out = config_bench(args.config, args, dev, stream, full=True)
    clk = clocks.stop()
    line = {"metric": out["metric"], "value": out["value"], "unit": "GUPS", "n_gpus": 1, "steps": None,
            "warmup": 1, "ms_per_step": out["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "clocks": clk,
            **{k: v for k, v in out.items() if k not in ("metric", "value", "ms_per_step", "unit", "dtype")}}
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args):
    """The reference arm: the reference's own CPU code on this host's cores (see
    cpu_reference_sample).  A step is one bounded sample; ms_per_step is its
    measured time, value the metric of the whole iteration it stands for."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    with c_stdout_to_stderr():
        inp = cpu_sample_inputs(args, threads)
        for _ in range(args.warmup):
            cpu_reference_sample(args, threads, inp)
        vals = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            vals.append(cpu_reference_sample(args, threads, inp))
        wall = time.perf_counter() - t0
    v = statistics.median(r["value"] for r in vals)
    last = vals[-1]
    line = {"impl": "reference", "metric": "projector GUPS over a 4D primal-dual iteration", "value": v,
            "unit": "GUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * statistics.median(r["sample_s"] for r in vals), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload(args),
            "cpu_baseline": {"value": v, "unit": "GUPS", "cores": last["cores"], "kind": last["kind"],
                             "sample": last["sample"]},
            "e2e": {"value": v, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "s_per_4d_pd_iter_extrapolated": statistics.median(r["s_per_iter"] for r in vals),
            "per_op_s": last["per_op_s"], "wall_s": wall}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def run_stt(args):
    import torch

    import spacetimetomography_b200 as stt

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        args.gpus = world if world > 1 else args.gpus
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from spacetimetomography_b200.halo import HaloExchange

    ctx, st, gmax, _ = build_problem(args, dev, rank)
    if world > 1:
        gmax_t = torch.tensor([gmax], device=dev)
        dist.all_reduce(gmax_t, op=dist.ReduceOp.MAX)
        gmax = float(gmax_t.item())
    F, V, N = args.frames, args.views, args.n
    pd = pd_params(gmax)
    bp_mode = 0 if args.bp == "voxel" else 1
    stream = torch.cuda.Stream(device=dev)
    halo = HaloExchange(rank, world, st, dist) if world > 1 else None

    def make_solver(mode):
        # the first solver tunes the context's launch choices (outside any timed region)
        return stt.Solver(ctx, st, F, V, pd, alpha=0.3, bp_mode=bp_mode, seed=99, mode=mode,
                          halo=(halo is not None and rank > 0), frame_offset=rank * F, total_frames=world * F,
                          autotune=True)

    solver = make_solver(stt.SOLVE_GRAPH)

    def step(s):
        if halo is not None:
            halo.exchange_xbar(stream)
            s.iterate_phase(0, stream)
            halo.exchange_duals(stream)
            s.iterate_phase(1, stream)
        else:
            s.iterate(1, stream)

    with torch.cuda.stream(stream):
        st["xbar"].copy_(st["vol"])
    for _ in range(args.warmup):
        step(solver)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step(solver)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    t = e0.elapsed_time(e1) / 1000.0
    if world > 1:
        tt = torch.tensor([t], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
        dist.barrier()
    t_iter = t / args.steps
    launches_per_iter, _ = solver.stats()
    value = world * F * N ** 3 * V / t_iter / 1e9

    # ---- dominant kernel: forward projection fused with the correction ----
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    corr = torch.empty((args.det, args.det), device=dev)
    rl = torch.zeros((args.det, args.det), device=dev)
    vol0 = st["vol"][0]
    with torch.cuda.stream(stream):
        for v in range(3):
            ctx.fp_correction(vol0, st["proj"][0, v], rl, corr, v, stream=stream)
        e2.record(stream)
        for v in range(V):
            ctx.fp_correction(vol0, st["proj"][0, v], rl, corr, v, stream=stream)
        e3.record(stream)
    torch.cuda.synchronize()
    t_fp = e2.elapsed_time(e3) / 1000.0 / V
    fp_bytes = 4 * N ** 3 + 12 * args.det * args.det  # volume read + b read, corr write, ray length (per view)
    peak, peak_kind = peaks()
    achieved = fp_bytes / t_fp / 1e9
    # samples per view and the gather ceiling over the same frame's views
    w = torch.zeros((1, args.det, args.det), device=dev)
    img = torch.zeros((1, args.det, args.det), device=dev)
    samples = 0.0
    for v in range(V):
        ctx.fp(vol0, img, view0=v, nviews=1, weight=w, stream=stream)
        torch.cuda.synchronize()
        samples += float(w.sum().item())
    gc = gather_ceilings(ctx, vol0, range(V), args.det, dev, stream)
    ceil = gc[gc["projector_fetch"]]["gsamples_per_s"]
    fp_samples = {"fp_s_per_view": t_fp, "samples_per_view": samples / V, "fp_gsamples_per_s": samples / V / t_fp / 1e9,
                  "gather_ceiling_gsamples_per_s": ceil, "gather_ceilings": gc,
                  "fp_frac_of_gather_ceiling": (samples / V / t_fp / 1e9) / ceil,
                  "views": f"the {V} views of frame 0, FP fused with the correction (stt_fp_correction, transposes "
                           "included); the gather ceiling is stt_gather_ceiling on the same views, in the corner "
                           "fetch the tuned projector uses (projector_fetch)"}

    # ---- the per-view GPU form ----
    plain = None
    if not args.no_plain and world == 1:
        sp = make_solver(stt.SOLVE_PLAIN)
        sp.iterate(1, stream)  # warm-up
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        sp.iterate(1, stream)
        p1.record(stream)
        torch.cuda.synchronize()
        plain = p0.elapsed_time(p1) / 1000.0
        sp.close()

    # ---- the persistent form: every frame's SART call in one cooperative launch ----
    persistent = None
    if not args.no_plain and world == 1 and bp_mode == 0:
        spp = make_solver(stt.SOLVE_PERSISTENT)
        spp.iterate(2, stream)  # warm-up (captures the iteration's graph)
        torch.cuda.synchronize()
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kq = max(1, min(args.steps, 5))
        q0.record(stream)
        spp.iterate(kq, stream)
        q1.record(stream)
        torch.cuda.synchronize()
        spp.poll_status(stream)
        blocks, graph = spp.persistent_info()
        t_p = q0.elapsed_time(q1) / 1000.0 / kq
        persistent = {"s_per_iter": t_p, "gups": F * N ** 3 * V / t_p / 1e9, "graph_vs_persistent": t_p / t_iter,
                      "blocks": blocks, "graph_captured": graph, "launches_per_iter": spp.stats()[0],
                      "note": "STT_SOLVE_PERSISTENT: warps, duals and primals as launches, then all frames' SART "
                              "calls, ROI masks and over-relaxations in one cooperative launch (k_sweep_persistent), "
                              "the same bits as the graph form; its gathers are plain loads (the texture path is "
                              "not coherent with the launch's own writes)"}
        spp.close()

    # ---- end to end with host buffers ----
    # Every step uploads its inputs (volumes, flows, projections) from pinned
    # host memory and reads its result back.  On one GPU this goes through the
    # host-buffer entry points of include/stt_host.h (stt_host_solver_*, the
    # call a host application makes): two slots, so step i+1's upload and step
    # i-1's read-back overlap step i's compute; every copy, the pipeline's fill
    # and its drain are inside the timed region (between two device events,
    # the host having waited for every step).
    host = {"vol": st["vol"][:F].detach().cpu().pin_memory(), "flow": st["flow"].detach().cpu().pin_memory(),
            "proj": st["proj"].detach().cpu().pin_memory()}
    h2d = sum(v.numel() * 4 for v in host.values())
    d2h = st["vol"][:F].numel() * 4
    ksteps = max(1, min(args.steps, 3))

    def reset_duals(s_):
        s_["xbar"].copy_(s_["vol"])
        for k_ in ("ytv", "ytp", "ybc"):
            s_[k_].zero_()

    if world == 1:
        from spacetimetomography_b200.host import HostSolver

        hs = HostSolver((N, N, N), (1.0, 1.0, 1.0), (args.det, args.det), 1.0, 600.0, 1000.0, angles_for(args, 0),
                        F, V, pd, alpha=0.3, bp_mode=bp_mode, seed=99, slots=2, device=local)
        outs = [torch.empty_like(st["vol"][:F], device="cpu").pin_memory() for _ in range(2)]
        for i in range(2):  # untimed: both slots capture their graphs here
            hs.submit(host["vol"], host["flow"], host["proj"], 1, outs[i % 2])
        while hs.pending():
            hs.wait()
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ksteps = max(1, args.steps)
        torch.cuda.synchronize()
        q0.record(stream)
        for i in range(ksteps):
            hs.submit(host["vol"], host["flow"], host["proj"], 1, outs[i % 2])
        while hs.pending():
            hs.wait()
        q1.record(stream)
        torch.cuda.synchronize()
        te = q0.elapsed_time(q1) / 1000.0
        hs.close()
    else:
        out_host = torch.empty_like(st["vol"][:F], device="cpu").pin_memory()

        def e2e_step():
            with torch.cuda.stream(stream):
                for k_, v_ in host.items():
                    st[k_].copy_(v_, non_blocking=True)
                reset_duals(st)
            step(solver)
            with torch.cuda.stream(stream):
                out_host.copy_(st["vol"][:F], non_blocking=True)

        e2e_step()
        torch.cuda.synchronize()
        dist.barrier()
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        for _ in range(ksteps):
            e2e_step()
        q1.record(stream)
        torch.cuda.synchronize()
        te = q0.elapsed_time(q1) / 1000.0
        tt = torch.tensor([te], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        te = float(tt.item())
    e2e_value = world * F * N ** 3 * V / (te / ksteps) / 1e9

    flow = None if args.no_flow else flow_bench(args, dev, stream, rank)

    # the single-frame workloads, one sub-line each (rank 0, one GPU)
    configs = None
    # config 4 (the batch of 64 uneven instances), a few iterations each form
    batch = None
    if not args.no_batch and world == 1:
        with c_stdout_to_stderr():
            batch = batch_leg(args, min(args.steps, 3), min(args.warmup, 2))
    if not args.no_configs and world == 1:
        configs = {}
        for cid in sorted(CONFIG_SPECS):
            try:
                configs[str(cid)] = config_bench(cid, args, dev, stream, rank)
            except Exception as e:  # a failing sub-line must not cost the headline line
                configs[str(cid)] = {"error": f"{type(e).__name__}: {e}"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        check = fp64_sart_check(ctx, st, args, gmax)
        with c_stdout_to_stderr():
            threads = os.cpu_count() or 1
            cpu = cpu_reference_sample(args, threads, cpu_sample_inputs(args, threads), gpu_check=check)
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_bind as ob

        with c_stdout_to_stderr():
            cpu["fp64_pd_iteration"] = fp64_pd_iteration_check(args, dev, stream, ob)

    if rank == 0:
        line = {"metric": "projector GUPS over a 4D primal-dual iteration", "value": value, "unit": "GUPS",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_iter,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": workload(args),
                "s_per_4d_pd_iter": t_iter,
                "plain_s_per_iter": plain,
                "batched_vs_plain": (plain / t_iter) if plain else None,
                "persistent": persistent,
                "roofline": {"bound": "hbm", "kernel": "k_fp_corr (forward projection + SART correction)",
                             "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                             "peak_source": peak_kind, "traffic": traffic_per_launch(args),
                             "algorithmic_bytes_per_launch": fp_bytes, "launch_s": t_fp,
                             "note": "volume is L2-resident; the kernel is bound by gather (L1/L2) throughput"},
                "fp_samples": fp_samples,
                "e2e": {"value": e2e_value, "unit": "GUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "through": ("stt_host_solver_submit/_wait (include/stt_host.h), 2 slots" if world == 1
                                    else "torch pinned copies around the sharded solver"),
                        "steps": ksteps},
                "gpu_launches": launches_per_iter * args.steps,
                "launches_per_iter": launches_per_iter,
                "tuning": ctx.get_tuning(),
                "clocks": clk,
                "cpu_baseline": None if cpu is None else {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "cpu_s_per_iter": None if cpu is None else cpu["s_per_iter"],
                "fp64_check": None if cpu is None else cpu.get("fp64_check"),
                "fp64_pd_iteration": None if cpu is None else cpu.get("fp64_pd_iteration"),
                "flow": flow,
                "configs": configs,
                "batch": batch}
        print(json.dumps(line), flush=True)
    solver.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_iter_probe(args) -> int:
    """The headline workload's solver (tuned, or with the choices --tuning
    names), one warm-up iteration, then one
    iteration inside the NVTX range "pd_iteration" and nothing else: the
    command whose launch list ncu records (--nvtx --nvtx-include
    "pd_iteration/")."""
    import torch

    import spacetimetomography_b200 as stt

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    ctx, st, gmax, _ = build_problem(args, dev, 0)
    stream = torch.cuda.Stream(device=dev)
    if args.tuning is not None:
        tune_or_set(ctx, stream, args.tuning)
    mode = stt.SOLVE_PERSISTENT if args.persistent else stt.SOLVE_GRAPH
    s = stt.Solver(ctx, st, args.frames, args.views, pd_params(gmax), alpha=0.3, bp_mode=0 if args.bp == "voxel" else 1,
                   seed=99, mode=mode, autotune=args.tuning is None and not args.persistent)
    with torch.cuda.stream(stream):
        st["xbar"].copy_(st["vol"])
    s.iterate(1, stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("pd_iteration")
    s.iterate(1, stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    s.poll_status(stream)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    s.iterate(1, stream)
    t1.record(stream)
    torch.cuda.synchronize()
    print(json.dumps({"launches_per_iter": s.stats()[0], "s_per_iter": t0.elapsed_time(t1) / 1000.0,
                      "persistent": s.persistent_info(), "tuning": ctx.get_tuning()}), flush=True)
    s.close()
    ctx.close()
    return 0


def run_flow_only(args):
    import torch

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    out = flow_bench(args, dev, stream, 0)
    line = {"metric": "optical-flow iterations (L1Huber_OF primal + dual)", "value": out["gvoxel_iter_per_s"],
            "unit": "Gvoxel-iterations/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic", "config": {"workload": out["workload"]}, **out}
    print(json.dumps(line), flush=True)
    return 0


def batch_fp64_check(inst, dev, stream, count=2) -> dict:
    """One primal-dual iteration of the batch's smallest instances (by voxels
    x views) against the FP64 oracle, FP32 and BF16 storage: each instance's
    own single-frame solve (which a batch reproduces bit for bit), from a
    state one GPU iteration into the solve, and the oracle's reference-ordered
    iteration (dual, primal, SART with voxel BP, ROI mask, over-relaxation)
    from the same state (for BF16 storage: the BF16 state, the oracle
    unrounded)."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200.api import REFERENCE_CUT

    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_bind as ob

    order = sorted(range(len(inst)), key=lambda k: inst[k]["geom"][0] ** 3 * inst[k]["proj"].shape[0])[:count]
    out = []
    for k in order:
        d = inst[k]
        n, det, ds, sid, sdd, ang = d["geom"]
        V = d["proj"].shape[0]
        pd = d["pd"]
        row = {"instance": k, "volume": n, "detector": det, "views": V}
        for storage in ("f32", "bf16"):
            dt = torch.bfloat16 if storage == "bf16" else torch.float32
            z = lambda *s_: torch.zeros(s_, device=dev)  # noqa: E731
            v0 = (0.8 * d["truth"]).to(dt)
            st = dict(vol=torch.stack([v0, v0]), xbar=torch.stack([v0, v0]), xprev=z(1, n, n, n).to(dt),
                      ytv=z(1, 3, n, n, n), ytp=z(1, n, n, n), ybc=z(1, n, n, n), flow=z(1, 3, n, n, n),
                      proj=d["proj"].to(dt).unsqueeze(0).contiguous())
            s1 = stt.Solver(d["ctx"], st, 1, V, pd, alpha=0.3, roi_cut=REFERENCE_CUT, seed=5, mode=stt.SOLVE_GRAPH,
                            storage=storage)
            s1.iterate(1, stream)  # into the solve: non-zero duals
            torch.cuda.synchronize()
            s1.close()
            start = {kk: vv.detach().float().cpu().numpy().copy() for kk, vv in st.items()}
            s2 = stt.Solver(d["ctx"], st, 1, V, pd, alpha=0.3, roi_cut=REFERENCE_CUT, seed=11, mode=stt.SOLVE_GRAPH,
                            storage=storage)
            s2.iterate(1, stream)
            torch.cuda.synchronize()
            s2.poll_status(stream)
            s2.close()
            gpu = st["vol"][0].float().cpu().numpy()
            pp = [pd.sigma, pd.tau, pd.tv_w, pd.tp_w, pd.bc_w, pd.huber_factor, pd.gmax]
            scan = ob.Scan(n, (det, det), sid=sid, sdd=sdd, ds=ds)
            with c_stdout_to_stderr():
                ref = ob.pd_iteration(scan, ang, start, 1, V, pp, tuple(pd.cut), REFERENCE_CUT, 0.3, 0,
                                      [stt.frame_order(11, 0, 1, 0, V)], [np.zeros((det, det), np.float64)],
                                      fp64=True)
            row[f"{storage}_vol_rel_l2_vs_fp64"] = ob.rel_l2(gpu, ref["vol"][0])
            del st
        out.append(row)
    return {"instances": out,
            "sample": "one PD iteration of each of the batch's two smallest instances (voxels x views) at its own "
                      "size, from one GPU iteration into the solve; relative L2 of the GPU volume against the FP64 "
                      "oracle (BF16 storage: the GPU's BF16 result against the unrounded FP64 iteration)"}


def run_batch_only(args):
    print(json.dumps(batch_leg(args, args.steps, args.warmup)), flush=True)
    return 0


def batch_leg(args, steps, warmup) -> dict:
    """Config 4: independent single-frame TV + SART solves of uneven size
    (cubes 64^3-192^3, detectors 128^2-384^2, 60-240 views, sid 500-700 mm,
    sdd 900-1100 mm, seeded), one batched graph iteration against the same
    instances solved one after another on one stream; `steps` timed
    iterations after `warmup`."""
    import torch

    import spacetimetomography_b200 as stt
    from spacetimetomography_b200 import phantom as ph

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(2024)
    inst, units = [], 0
    for k in range(args.batch_instances):
        n = int(rng.integers(64, 193))
        det = int(rng.integers(128, 385))
        V = int(rng.integers(60, 241))
        sid, sdd = float(rng.uniform(500, 700)), float(rng.uniform(900, 1100))
        dims = (n, n, n)
        ang = np.sort(rng.uniform(0, 2 * math.pi, V))
        ctx = stt.Context(0)
        # detector pixel size covering the magnified volume
        ds = max(1.0, 1.1 * n * sdd / sid / det)
        ctx.set_geometry(dims, (1.0, 1.0, 1.0), (det, det), ds, sid, sdd, ang)
        truth = ph.ellipsoid_phantom(dims, 12, seed=100 + k, semi=(0.04 * n, 0.3 * n), device=dev)
        proj = torch.zeros((V, det, det), device=dev)
        ctx.fp(truth, proj)
        torch.cuda.synchronize()
        pd = stt.PdParams(tv_w=0.01, tp_w=0.0, bc_w=0.0, huber_factor=float(1 / (1 + 0.1125)),
                          gmax=float(proj.max().item() / 4))
        inst.append(dict(ctx=ctx, vol=torch.zeros_like(truth), proj=proj, bp_mode=0, alpha=0.3, pd=pd, seed=k,
                         truth=truth, geom=(n, det, ds, sid, sdd, ang)))
        units += n ** 3 * V
    stream = torch.cuda.Stream(device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    staging = {}

    def batched_time():
        for d in inst:
            d["vol"].zero_()
        b = stt.Batch(inst, mode=stt.SOLVE_GRAPH)
        staging["f32"] = b.staging()
        for _ in range(warmup):
            b.iterate(1, stream)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            b.iterate(1, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        b.close()
        return e0.elapsed_time(e1) / 1000.0 / steps

    t_default = batched_time()  # the default launch choices
    t0 = time.perf_counter()
    choices = [d["ctx"].autotune(stream) for d in inst]  # every instance's own geometry
    for d in inst:
        d["autotune"] = True  # the batch then also chooses its projector split as a whole (stt_batch_staging)
    t_tune = time.perf_counter() - t0
    t_batch = batched_time()
    f32_result = [d["vol"].clone() for d in inst]
    # BF16 storage of the same instances (volumes and sinograms in BF16, FP32
    # arithmetic), the same iterations from the same start
    inst16 = [dict(d, vol=torch.zeros_like(d["vol"], dtype=torch.bfloat16), proj=d["proj"].to(torch.bfloat16),
                   storage="bf16") for d in inst]
    for d in inst16:
        d.pop("truth")
    b16 = stt.Batch(inst16, mode=stt.SOLVE_GRAPH)
    staging["bf16"] = b16.staging()
    for _ in range(warmup):
        b16.iterate(1, stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        b16.iterate(1, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_b16 = e0.elapsed_time(e1) / 1000.0 / steps
    b16.close()
    num = sum(float((d["vol"].float() - r).norm() ** 2) for d, r in zip(inst16, f32_result))
    den = sum(float(r.norm() ** 2) for r in f32_result)
    bf16_vs_f32 = math.sqrt(num / den)
    bf16_err = [float((d["vol"].float() - o["truth"]).norm() / o["truth"].norm()) for d, o in zip(inst16[:4], inst)]
    del inst16
    # every instance's SART call in ONE persistent cooperative launch per
    # iteration (STT_SOLVE_PERSISTENT), the same iterations from the same start
    for d in inst:
        d["vol"].zero_()
    bpers = stt.Batch(inst, mode=stt.SOLVE_PERSISTENT)
    for _ in range(warmup):
        bpers.iterate(1, stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        bpers.iterate(1, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    bpers.poll_status(stream)
    t_pers = e0.elapsed_time(e1) / 1000.0 / steps
    bpers.close()
    pers_diff = max(float((d["vol"] - r).abs().max()) for d, r in zip(inst, f32_result))
    # the instances' own tuned choices again (the batches may have set their
    # staged masks to 0), for the one-after-another forms below
    for d, c in zip(inst, choices):
        d["ctx"].set_tuning(c["fp_variant"], c["slab_variant"], c["bp_variant"], staged_bins=c["staged_bins"],
                            ray_variant=c["ray_variant"], staged_bins_bf16=c["staged_bins_bf16"])
    # the same instances one after another (each its own graph-captured solver)
    solvers = []
    for d in inst:
        n3 = d["vol"].shape
        st = dict(vol=torch.zeros((2,) + n3, device=dev), xbar=torch.zeros((2,) + n3, device=dev),
                  xprev=torch.zeros((1,) + n3, device=dev), ytv=torch.zeros((1, 3) + n3, device=dev),
                  ytp=torch.zeros((1,) + n3, device=dev), ybc=torch.zeros((1,) + n3, device=dev),
                  flow=torch.zeros((1, 3) + n3, device=dev), proj=d["proj"].unsqueeze(0))
        solvers.append((stt.Solver(d["ctx"], st, 1, d["proj"].shape[0], d["pd"], alpha=0.3, seed=d["seed"],
                                   mode=stt.SOLVE_GRAPH), st))
    for sv, _ in solvers:
        sv.iterate(1, stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for sv, _ in solvers:
        sv.iterate(1, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_seq = e0.elapsed_time(e1) / 1000.0
    # the same instances in the plain per-view form (every view's launches
    # from the host loop, a host synchronisation after each view), one after
    # another: the form batching replaces
    plain = []
    for d, (_, st) in zip(inst, solvers):
        plain.append(stt.Solver(d["ctx"], st, 1, d["proj"].shape[0], d["pd"], alpha=0.3, seed=d["seed"],
                                mode=stt.SOLVE_PLAIN))
    for sv in plain[:2]:
        sv.iterate(1, stream)  # warm-up
    torch.cuda.synchronize()
    e0.record(stream)
    for sv in plain:
        sv.iterate(1, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1) / 1000.0
    for sv in plain:
        sv.close()
    errs = [float((d["vol"] - d["truth"]).norm() / d["truth"].norm()) for d in inst[:4]]
    fp64 = batch_fp64_check(inst, dev, stream)
    line = {"metric": "projector GUPS over one batched iteration of independent instances", "value": units / t_batch / 1e9,
            "unit": "GUPS", "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": 1000 * t_batch,
            "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.batch_instances} single-frame TV + SART instances, cubes 64^3-192^3, "
                                   "detectors 128^2-384^2, 60-240 views, voxel-based BP"},
            "sequential_ms_per_iter": 1000 * t_seq, "batched_vs_sequential": t_seq / t_batch,
            "plain_ms_per_iter": 1000 * t_plain, "batched_vs_plain": t_plain / t_batch,
            "plain_note": "the same instances one after another in the per-view form (STT_SOLVE_PLAIN: each "
                          "view's launches from a host loop, a host synchronisation per view)",
            "rel_l2_to_phantom_first4": errs,
            "fp64_check": fp64,
            "persistent": {"ms_per_iter": 1000 * t_pers, "gups": units / t_pers / 1e9,
                           "graph_vs_persistent": t_pers / t_batch, "max_abs_diff_to_graph_batch": pers_diff,
                           "note": "STT_SOLVE_PERSISTENT: every instance's duals and primal on its stream, then all "
                                   "64 SART calls in one cooperative launch (blocks split by work)"},
            "bf16_storage": {"ms_per_iter": 1000 * t_b16, "gups": units / t_b16 / 1e9,
                             "rel_l2_to_f32_storage": bf16_vs_f32, "rel_l2_to_phantom_first4": bf16_err,
                             "iterations": warmup + steps,
                             "note": "volumes and sinograms stored in BF16, FP32 arithmetic; compared with the "
                                     "FP32-storage batch after the same iterations from the same start"},
            "autotune": {"batched_ms_per_iter_default_choices": 1000 * t_default,
                         "batched_ms_per_iter_tuned": 1000 * t_batch, "tuned_vs_default": t_default / t_batch,
                         "tuning_s_all_instances": t_tune,
                         "batch_staging": staging,
                         "cache_hits": sum(c["from_cache"] for c in choices),
                         "fp_variant_counts": np.bincount([c["fp_variant"] for c in choices], minlength=10).tolist(),
                         "slab_variant_counts": np.bincount([c["slab_variant"] for c in choices], minlength=8).tolist(),
                         "bp_variant_counts": np.bincount([c["bp_variant"] for c in choices], minlength=5).tolist(),
                         "first_instances": [{k: c[k] for k in ("fp", "slab", "bp", "staged_bins")}
                                             for c in choices[:4]]}}
    for sv, _ in solvers:
        sv.close()
    return line


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.config is not None:
        return run_config_only(args)
    if args.flow_only:
        return run_flow_only(args)
    if args.batch_only:
        return run_batch_only(args)
    if args.iter_probe:
        return run_iter_probe(args)
    if args.fp64_pd_check:
        import torch

        torch.cuda.set_device(0)
        dev = torch.device("cuda", 0)
        sys.path.insert(0, str(ROOT / "tests"))
        import oracle_bind as ob

        with c_stdout_to_stderr():
            out = fp64_pd_iteration_check(args, dev, torch.cuda.Stream(device=dev), ob)
        print(json.dumps({"fp64_pd_iteration": out}), flush=True)
        return 0
    return run_stt(args)


if __name__ == "__main__":
    sys.exit(main())
