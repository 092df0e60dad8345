#!/usr/bin/env python
"""Headline benchmark of the B200 particle locate + link engine.

Workload (one step = one pass of the hot path over one synthetic video):
2000 frames of 2048x2048 uint16, 2000 Gaussian spots per frame (sigma uniform
1.2-2.5 px, peak SNR log-normal in 3-20 over a background of 100 with
Poisson noise), Brownian motion D = 1.0 px^2/frame with 2 % births/deaths per
frame; trackpy-style locate with diameter 11, full characterization and the
doughnut correction (the Python defaults), minmass 220 (the configuration
names none; 220 separates the noise maxima, mass <= 190, from the dimmest
true spots, mass >= 260, on this generator), linking with search_range 7 and
memory 3.  The video is generated on the device and stays in HBM (16.8 GB,
larger than L2, so no flush is needed between steps).

  value  frames/s over all ranks, inputs resident in HBM, device-timed with
         CUDA events (max over ranks)
  e2e    the same through the public Python API (gt.batch on a pinned host
         array, host->device copies and the DataFrame read-back included)

Multi-GPU (torchrun): weak scaling, every rank tracks its own video (frames
and videos are independent; no data-path collective).

`--impl reference` times the CPU restatement of the reference's path (the
oracle; the reference's own Rust/wgpu build is unavailable here) on the host
cores with every thread, on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "frames/s + features/s at 2048²: plain vs learned-proposal; % HBM roofline"
CONFIG = dict(workload="plain batch locate+characterize+link, 2000 frames 2048x2048 uint16, 2000 spots/frame",
              frames=2000, height=2048, width=2048, spots_per_frame=2000, diameter=11, minmass=220.0,
              separation=12, characterize=True, doughnut_correction=True, search_range=7.0, memory=3,
              sigma_px=[1.2, 2.5], snr=[3, 20], background=100, D=1.0, births_deaths=0.02,
              l2="inputs (16.8 GB) larger than L2; no flush", style="trackpy")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--frames", type=int, default=CONFIG["frames"])
    ap.add_argument("--size", type=int, default=CONFIG["height"])
    ap.add_argument("--cpu-sample", type=int, default=0, help="frames in the CPU-baseline sample (0: auto)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--workload", default="headline", choices=["headline", "ragged", "learned", "log"],
                    help="headline: the 2000-frame 2048^2 video; ragged: 64 videos of uneven size and length; "
                         "learned: plain vs learned-proposal seeds on 1000 frames of 2048^2 at 4000 spots/frame; "
                         "log: multi-scale LoG on 500 frames of 1024^2 float32")
    ap.add_argument("--learned-scale", type=float, default=1.0, help="learned: fraction of the 1000 frames timed")
    ap.add_argument("--epochs", type=float, default=3.0, help="learned: passes over the 200k training crops")
    ap.add_argument("--train-frames", type=int, default=800, help="learned: labelled frames the crops come from")
    ap.add_argument("--scale", type=float, default=0.25,
                    help="ragged: fraction of the configured 50-1000 frames per video")
    return ap.parse_args()


def params():
    from gpu_tracking_b200._params import trackpy_params
    return trackpy_params(CONFIG["diameter"], minmass=CONFIG["minmass"], search_range=CONFIG["search_range"],
                          memory=CONFIG["memory"])


def make_video(n_frames, size, seed, device):
    from gpu_tracking_b200.synth import brownian_video
    return brownian_video(n_frames, size, size, CONFIG["spots_per_frame"], seed=seed, device=device,
                          sigma_range=tuple(CONFIG["sigma_px"]), snr_range=tuple(CONFIG["snr"]),
                          bg=CONFIG["background"], D=CONFIG["D"], turnover=CONFIG["births_deaths"])


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_issue():
    """Thread-instructions per pixel of the dominant kernel from the committed
    ncu summary (profiles/issue.json)."""
    try:
        with open(os.path.join(ROOT, "profiles", "issue.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def load_traffic():
    """Per-frame DRAM traffic of the dominant kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample_frames(cores, total):
    """Frames in the CPU sample: about 10-20 s of oracle work on the host's cores
    (the oracle locates ~1.3 frames/s per core at 2048x2048)."""
    return max(16, min(total, 256, 16 * cores))


def cpu_baseline(frames_u16, p, nthreads):
    """The oracle on the host cores; returns frames/s and the sample size."""
    import numpy as np
    from oracle import loader
    f32 = frames_u16.astype(np.float32)
    t = time.perf_counter()
    tab = loader.batch(p, f32, nthreads=nthreads)
    dt = time.perf_counter() - t
    return len(f32) / dt, dt, len(tab)


def run_reference(args):
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import torch
    dev = "cuda:0" if torch.cuda.is_available() else "cpu"
    cores = os.cpu_count() or 1
    n = args.cpu_sample or cpu_sample_frames(cores, args.frames)
    vid = make_video(n, args.size, 2, dev).cpu().numpy()
    p = params()
    vals = []
    for i in range(args.warmup + args.steps):
        fps, dt, rows = cpu_baseline(vid, p, cores)
        if i >= args.warmup:
            vals.append(fps)
    v = statistics.median(vals)
    sample = "%d frames of the %dx%d workload (oracle, locate+characterize+doughnut with %d threads, link serial)" % (
        n, args.size, args.size, cores)
    line = {"metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * n / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": dict(CONFIG, frames=n, height=args.size, width=args.size, parallelism="host threads"),
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


RAGGED = dict(workload="64 ragged uint16 videos: sides in {256,512,1024,1536,2048}, 50-1000 frames (x scale), "
                        "density 1e-4..2e-3 spots/px^2, D 0.2..2", videos=64, diameter=11, minmass=220.0,
              search_range=7.0, memory=3, seed=4)


def ragged_videos(scale, device):
    """The 64 videos of the ragged workload, generated on the device."""
    import numpy as np
    from gpu_tracking_b200.synth import brownian_video
    rng = np.random.default_rng(RAGGED["seed"])
    vids = []
    for k in range(RAGGED["videos"]):
        H = int(rng.choice([256, 512, 1024, 1536, 2048]))
        W = int(rng.choice([256, 512, 1024, 1536, 2048]))
        T = max(1, int(rng.integers(50, 1001) * scale))
        n = max(1, int(rng.uniform(1e-4, 2e-3) * H * W))
        D = float(rng.uniform(0.2, 2.0))
        vids.append(brownian_video(T, H, W, n, seed=1000 + k, device=device, D=D))
    return vids


def run_ragged(args):
    """Frames/s of the ragged workload through gt_batch_videos (device-resident),
    beside the same videos through one gt_batch call each."""
    import ctypes

    import torch
    from gpu_tracking_b200 import _ffi
    from gpu_tracking_b200._params import DTYPE_U16, trackpy_params
    torch.cuda.set_device(0)
    vids = ragged_videos(args.scale, "cuda:0")
    torch.cuda.synchronize()
    p = trackpy_params(RAGGED["diameter"], minmass=RAGGED["minmass"], search_range=RAGGED["search_range"],
                       memory=RAGGED["memory"])
    ctx = _ffi.context(0)
    L = _ffi.lib()
    n = len(vids)
    vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32
    ptrs = (vp * n)(*[v.data_ptr() for v in vids])
    Ts = (i64 * n)(*[v.shape[0] for v in vids])
    Hs = (i32 * n)(*[v.shape[1] for v in vids])
    Ws = (i32 * n)(*[v.shape[2] for v in vids])
    frames = sum(v.shape[0] for v in vids)
    pixels = sum(v.numel() for v in vids)

    def together():
        outs = (vp * n)()
        ctx.check(L.gt_batch_videos(ctx.handle, ctypes.byref(p), n, ptrs, DTYPE_U16, Ts, Hs, Ws, outs))
        rows = 0
        for i in range(n):
            rows += L.gt_table_nrows(outs[i])
            L.gt_table_free(outs[i])
        return rows

    def loop():
        rows = 0
        for v in vids:
            out = vp()
            ctx.check(L.gt_batch(ctx.handle, ctypes.byref(p), vp(v.data_ptr()), DTYPE_U16, v.shape[0], v.shape[1],
                                 v.shape[2], None, None, 0, ctypes.byref(out)))
            rows += L.gt_table_nrows(out)
            L.gt_table_free(out)
        return rows

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        rows = 0
        for _ in range(args.steps):
            rows = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps, rows

    clocks = Clocks(0)
    clocks.start()
    n0 = ctx.launch_count()
    ms, rows = timed(together)
    launches = (ctx.launch_count() - n0) // (args.warmup + args.steps)
    clk = clocks.stop()
    ms_loop, rows_loop = timed(loop)
    if rows != rows_loop:
        raise SystemExit("gt_batch_videos found %d rows, the gt_batch loop %d" % (rows, rows_loop))
    # where one call's time goes: device time of the stages, host time of the phases
    ctx.profile(True)
    together()
    parts = {}
    for name in ("bandpass_localmax", "walk_characterize", "finalize", "scatter", "link_sort", "link_lists",
                 "link_video", "link_durations", "round_ids", "host_locate", "host_assemble", "host_link"):
        k, kms = ctx.profile_read(name)
        if k:
            parts[name] = {"count": k, "ms": kms}
    ctx.profile(False)
    # the wave shape the autotuner chose (tile rows, processed bytes per wave)
    L.gt__ragged_shape.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i64)]
    seg, budget = i32(), i64()
    L.gt__ragged_shape(ctx.handle, ctypes.byref(seg), ctypes.byref(budget))
    line = {"metric": "frames/s, 64 ragged videos (one gt_batch_videos call)", "value": frames / (ms / 1000.0),
            "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(RAGGED, scale=args.scale, frames=frames, pixels=pixels,
                           l2="inputs (%.1f GB) larger than L2; no flush" % (pixels * 2 / 1e9)),
            "features_per_s": rows / (ms / 1000.0), "features": rows,
            "loop_of_gt_batch": {"value": frames / (ms_loop / 1000.0), "ms_per_step": ms_loop},
            "profile_one_call": parts,
            "tuned_wave_shape": {"tile_rows": seg.value, "wave_bytes": budget.value},
            "gpu_launches": launches, "clocks": clk}
    print(json.dumps(line))
    return 0


LEARNED = dict(workload="plain vs learned-proposal seeds: 1000 frames 2048x2048 uint16, 4000 spots/frame, SNR 2-10",
               frames=1000, size=2048, spots_per_frame=4000, snr=[2, 10], sigma_px=[1.2, 2.5], background=100,
               D=1.0, births_deaths=0.02, diameter=11, minmass=220.0, search_range=7.0, memory=3,
               net="4 x conv3x3 over 4x4-pixel cells: 16-32-32-32-3 channels, 24003 parameters, BF16/FP32 accumulate",
               train="200k crops of 128x128 (782 steps of 256 per epoch) from 800 frames of the 2000-spot SNR 3-20 "
                     "generator, labelled by the plain method's detections",
               calibration="8 held-out frames of the 4000-spot SNR 2-10 generator, recall target 0.997")


def cnn_flops_per_cell():
    """Multiply-adds x 2 of the four convolutions per 4x4-pixel cell."""
    return 2 * 9 * (16 * 32 + 32 * 32 + 32 * 32 + 32 * 3)


def run_learned(args):
    """Plain and learned-seed tracking of the same device-resident video."""
    import ctypes

    import numpy as np
    import torch
    import gpu_tracking_b200 as gt
    from gpu_tracking_b200 import _ffi, learned
    from gpu_tracking_b200._params import DTYPE_U16, trackpy_params
    from gpu_tracking_b200.synth import brownian_video
    torch.cuda.set_device(0)
    cfg = LEARNED
    S = cfg["size"]
    T = max(4, int(cfg["frames"] * args.learned_scale))
    epochs = args.epochs
    gen = dict(sigma_range=tuple(cfg["sigma_px"]), bg=cfg["background"], D=cfg["D"], turnover=cfg["births_deaths"])

    # training: frames of the 2000-spot generator labelled by the plain method
    t_start = time.perf_counter()
    train = brownian_video(args.train_frames, S, S, 2000, seed=101, device="cuda:0", snr_range=(3.0, 20.0), **gen)
    labels = gt.batch(train, cfg["diameter"], minmass=cfg["minmass"], tqdm=False)
    net = learned.ProposalNet(seed=1)
    net.fit_normalization(train)
    steps = int(round(epochs * 200_000 / 256))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = net.train(train, labels, steps=steps, batch=256, crop=128, lr=3e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del train, labels
    torch.cuda.empty_cache()
    calib = brownian_video(8, S, S, cfg["spots_per_frame"], seed=202, device="cuda:0",
                           snr_range=tuple(cfg["snr"]), **gen)
    thr, curve = learned.calibrate(net, calib, cfg["diameter"], recall=0.997, minmass=cfg["minmass"])
    del calib
    setup_s = time.perf_counter() - t_start

    video = brownian_video(T, S, S, cfg["spots_per_frame"], seed=303, device="cuda:0",
                           snr_range=tuple(cfg["snr"]), **gen)
    torch.cuda.synchronize()
    p = trackpy_params(cfg["diameter"], minmass=cfg["minmass"], search_range=cfg["search_range"],
                       memory=cfg["memory"])
    ctx = _ffi.context(0)
    L = _ffi.lib()

    def call(fn):
        out = ctypes.c_void_p()
        ctx.check(fn(ctypes.byref(out)))
        n = L.gt_table_nrows(out)
        L.gt_table_free(out)
        return n

    def plain_call(out):
        return L.gt_batch(ctx.handle, ctypes.byref(p), ctypes.c_void_p(video.data_ptr()), DTYPE_U16, T, S, S, None,
                          None, 0, out)

    def learned_call(out):
        return L.gt_batch_learned(ctx.handle, ctypes.byref(p), net.handle, ctypes.c_void_p(video.data_ptr()),
                                  DTYPE_U16, T, S, S, None, None, 0, out)

    def timed(fn, names):
        for _ in range(args.warmup):
            call(fn)
        torch.cuda.synchronize()
        starts = L.gt_last_walk_starts(ctx.handle)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        rows = 0
        for _ in range(args.steps):
            rows += call(fn)
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / args.steps
        # kernel times from one more, profiled call
        ctx.profile(True)
        l0 = ctx.launch_count()
        call(fn)
        launches = ctx.launch_count() - l0
        kern = {}
        for k in names:
            n, kms = ctx.profile_read(k)
            if n:
                kern[k] = {"launches": n, "ms": kms}
        ctx.profile(False)
        return ms, rows / args.steps, starts, kern, launches

    common = ("finalize", "scatter", "link_video", "link_lists", "link_sort", "link_rows")
    clocks = Clocks(0)
    clocks.start()
    ms_p, rows_p, starts_p, kern_p, launches_p = timed(plain_call, ("bandpass_localmax", "walk_characterize") + common)
    ms_l, rows_l, starts_l, kern_l, launches_l = timed(learned_call, ("proposal_net", "walk_local") + common)
    clk = clocks.stop()
    kw = dict(minmass=cfg["minmass"], search_range=cfg["search_range"], memory=cfg["memory"], tqdm=False)
    score = learned.compare(gt.batch(video, cfg["diameter"], **kw),
                            learned.batch_learned(video, cfg["diameter"], net, **kw))
    # the locate stage alone (no linking): where the seeds replace the bandpass local maxima
    p_loc = trackpy_params(cfg["diameter"], minmass=cfg["minmass"])

    def plain_loc(out):
        return L.gt_batch(ctx.handle, ctypes.byref(p_loc), ctypes.c_void_p(video.data_ptr()), DTYPE_U16, T, S, S,
                          None, None, 0, out)

    def learned_loc(out):
        return L.gt_batch_learned(ctx.handle, ctypes.byref(p_loc), net.handle, ctypes.c_void_p(video.data_ptr()),
                                  DTYPE_U16, T, S, S, None, None, 0, out)

    ms_pl, _, _, _, _ = timed(plain_loc, ())
    ms_ll, _, _, _, _ = timed(learned_loc, ())

    pk = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
    except Exception:
        pass
    # the network runs inside a long step: the sustained GEMM figure when measured
    tc_peak = float(pk.get("bf16_tflops_sustained", pk.get("bf16_tflops", 1590.0)))
    net_ms = kern_l.get("proposal_net", {}).get("ms")
    flops = cnn_flops_per_cell() * ((S + 3) // 4) ** 2 * T
    tensor = None
    if net_ms:
        achieved = flops / (net_ms / 1000.0) / 1e12
        tensor = {"bound": "tensor", "achieved": achieved, "peak": tc_peak, "unit": "TFLOP/s",
                  "frac": achieved / tc_peak, "kernel": "proposal_net (4 conv3x3 launches per frame group)",
                  "flops_per_frame": flops / T, "peak_kind": "measured" if pk else "fallback"}
    hbm_peak, hbm_kind = load_peaks()
    bytes_per_frame_p = S * S * 2 + rows_p / T * 48.0
    bytes_per_frame_l = S * S * 2 + rows_l / T * 48.0
    line = {"metric": METRIC, "value": T / (ms_l / 1000.0), "unit": "frames/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_l, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 network, f32 walk", "data": "synthetic",
            "config": dict(cfg, frames=T, epochs=epochs, train_steps=steps, train_frames=args.train_frames,
                           l2="inputs (%.1f GB) larger than L2; no flush" % (T * S * S * 2 / 1e9)),
            "features_per_s": rows_l / (ms_l / 1000.0),
            "plain": {"value": T / (ms_p / 1000.0), "ms_per_step": ms_p, "features_per_s": rows_p / (ms_p / 1000.0),
                      "walk_starts": int(starts_p), "kernels": kern_p, "gpu_launches": int(launches_p),
                      "hbm_frac_whole_step": T * bytes_per_frame_p / (ms_p / 1000.0) / 1e9 / hbm_peak},
            "learned": {"value": T / (ms_l / 1000.0), "ms_per_step": ms_l, "features_per_s": rows_l / (ms_l / 1000.0),
                        "walk_starts": int(starts_l), "kernels": kern_l, "gpu_launches": int(launches_l),
                        "hbm_frac_whole_step": T * bytes_per_frame_l / (ms_l / 1000.0) / 1e9 / hbm_peak,
                        "threshold": thr, "calibration": curve},
            "speedup_learned_over_plain": ms_p / ms_l,
            "locate_only": {"plain": T / (ms_pl / 1000.0), "learned": T / (ms_ll / 1000.0), "unit": "frames/s",
                            "speedup_learned_over_plain": ms_pl / ms_ll},
            "score_vs_plain": score,
            "training": {"steps": steps, "seconds": train_s, "loss_first": loss[:20].mean(0).tolist(),
                         "loss_last": loss[-20:].mean(0).tolist(), "setup_seconds": setup_s},
            "roofline": tensor, "hbm_peak": hbm_peak, "hbm_peak_kind": hbm_kind,
            "gpu_launches": int(launches_l), "clocks": clk}
    print(json.dumps(line))
    return 0


LOG = dict(workload="multi-scale LoG detect+characterize+link, 500 frames 1024x1024 float32, 1500 blobs/frame",
           frames=500, height=1024, width=1024, blobs_per_frame=1500, radius_px=[2.0, 8.0], read_noise=5.0,
           background=50.0, snr=[3, 20], D=1.0, births_deaths=0.02, min_radius=2.0, max_radius=8.0, n_radii=10,
           log_spacing=True, minmass=150.0, characterize=True, doughnut_correction=True, search_range=6.0,
           memory=0, style="log", seed=3)


def log_taps_per_pixel(p):
    """Taps of the four separable passes of every radius, per pixel: each
    radius r filters with 2*rint+1 taps, rint = int(4 r / sqrt(2) + 0.5)
    (separable_log.wgsl), in each of its four passes."""
    import math
    import numpy as np
    n = int(p.n_radii)
    if p.log_spacing:
        radii = np.logspace(math.log10(p.min_radius), math.log10(p.max_radius), n).astype(np.float32)
    else:
        radii = np.linspace(p.min_radius, p.max_radius, n).astype(np.float32)
    return sum(4 * (2 * int(4.0 * float(r / np.float32(math.sqrt(2.0))) + 0.5) + 1) for r in radii)


def run_log(args):
    """Frames/s of the LoG workload, video resident in HBM, with an FP32
    roofline of the scale-space kernel (its tap multiply-adds per frame)."""
    import ctypes

    import torch
    from gpu_tracking_b200 import _ffi
    from gpu_tracking_b200._params import DTYPE_F32, log_params
    from gpu_tracking_b200.synth import blob_video
    torch.cuda.set_device(0)
    cfg = LOG
    T = args.frames if args.frames != CONFIG["frames"] else cfg["frames"]
    H = W = args.size if args.size != CONFIG["height"] else cfg["height"]
    video = blob_video(T, H, W, cfg["blobs_per_frame"], seed=cfg["seed"], device="cuda:0",
                       radius_range=tuple(cfg["radius_px"]), read_noise=cfg["read_noise"], bg=cfg["background"],
                       snr_range=tuple(cfg["snr"]), D=cfg["D"], turnover=cfg["births_deaths"])
    torch.cuda.synchronize()
    p = log_params(cfg["min_radius"], cfg["max_radius"], n_radii=cfg["n_radii"], log_spacing=cfg["log_spacing"],
                   minmass=cfg["minmass"], search_range=cfg["search_range"])
    ctx = _ffi.context(0)
    L = _ffi.lib()

    def step():
        out = ctypes.c_void_p()
        ctx.check(L.gt_batch(ctx.handle, ctypes.byref(p), ctypes.c_void_p(video.data_ptr()), DTYPE_F32, T, H, W,
                             None, None, 0, ctypes.byref(out)))
        n = L.gt_table_nrows(out)
        L.gt_table_free(out)
        return n

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.start()
    ctx.profile(True)
    l0 = ctx.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    rows = 0
    for _ in range(args.steps):
        rows += step()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launch_count() - l0
    kernels = {}
    for name in ("bandpass", "log_scale_space", "laplace", "logspace_max", "walk_characterize", "finalize", "scatter", "link_sort",
                 "link_lists", "link_video", "link_rows"):
        n, kms = ctx.profile_read(name)
        if n:
            kernels[name] = (n, kms)
    ctx.profile(False)
    clk = clocks.stop()
    frames = T * args.steps
    taps = log_taps_per_pixel(p)
    flops_per_frame = 2.0 * taps * H * W
    # FP32 peak: no measured figure exists for CUDA-core FP32, so the nominal
    # one at the sampled SM clock: 148 SMs x 128 FP32 lanes x 2 flops
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    fused = "log_scale_space" in kernels
    lap = kernels.get("log_scale_space") or kernels.get("laplace")
    roofline = None
    if lap:
        achieved = flops_per_frame * frames / (lap[1] / 1000.0) / 1e12
        tr = load_traffic().get("log_scale_space", {}) if fused else {}
        roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp32_peak,
                    "kernel": "log_scale_space (all radii and the 3-D maximum)" if fused else "laplace",
                    "peak_kind": "nominal: 148 SMs x 128 FP32 lanes x 2 flops at the sampled SM clock",
                    "flops_per_frame": flops_per_frame, "taps_per_pixel": taps,
                    "traffic": tr.get("dram_bytes_per_frame"), "traffic_source": tr.get("source")}
    hbm_peak, hbm_kind = load_peaks()
    total_k = sum(v[1] for v in kernels.values()) or 1.0
    line = {"metric": "frames/s, multi-scale LoG 1024x1024 float32 (10 radii), detect+characterize+link",
            "value": frames / (ms / 1000.0), "unit": "frames/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(cfg, frames=T, height=H, width=W,
                           l2="inputs (%.1f GB) larger than L2; no flush" % (T * H * W * 4 / 1e9)),
            "features_per_s": rows / (ms / 1000.0), "features_per_frame": rows / frames,
            "gpu_launches": int(launches), "roofline": roofline,
            "hbm": {"algorithmic_bytes_per_frame": H * W * 4 + rows / frames * 52.0, "peak": hbm_peak,
                    "peak_kind": hbm_kind,
                    "whole_step_frac": frames * (H * W * 4 + rows / frames * 52.0) / (ms / 1000.0) / 1e9 / hbm_peak},
            "kernel_ms_per_frame": {k: v[1] / frames for k, v in kernels.items()},
            "kernel_share": {k: round(v[1] / total_k, 4) for k, v in kernels.items()},
            "clocks": clk}
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ragged":
        return run_ragged(args)
    if args.workload == "learned":
        return run_learned(args)
    if args.workload == "log":
        return run_log(args)
    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    os.environ["GT_DEVICE"] = str(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()

    import gpu_tracking_b200 as gt
    from gpu_tracking_b200 import _ffi
    from gpu_tracking_b200._params import DTYPE_U16

    T, S = args.frames, args.size
    video = make_video(T, S, 2 + rank, "cuda:%d" % local)
    torch.cuda.synchronize()
    p = params()
    ctx = _ffi.context(local)
    L = _ffi.lib()

    def step():
        out = ctypes.c_void_p()
        ctx.check(L.gt_batch(ctx.handle, ctypes.byref(p), ctypes.c_void_p(video.data_ptr()), DTYPE_U16, T, S, S,
                             None, None, 0, ctypes.byref(out)))
        n = L.gt_table_nrows(out)
        L.gt_table_free(out)
        return n

    for _ in range(args.warmup):
        rows = step()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ctx.profile(True)
    l0 = ctx.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    ev0.record()
    rows_total = 0
    for _ in range(args.steps):
        rows_total += step()
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launch_count() - l0
    # local-maximum candidates the walk started from in the last call (noise maxima included)
    cands_per_frame = L.gt_last_walk_starts(ctx.handle) / float(T)
    kernels = {}
    for name in ("bandpass_localmax", "walk_characterize", "finalize", "scatter", "link_sort", "link_lists",
                 "link_video", "link_rows", "link_durations", "round_ids"):
        n, kms = ctx.profile_read(name)
        if n:
            kernels[name] = (n, kms)
    ctx.profile(False)
    clk = clocks.stop()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        r = torch.tensor([rows_total], device="cuda", dtype=torch.float64)
        dist.all_reduce(r)
        rows_all = float(r.item())
    else:
        rows_all = float(rows_total)
    frames_all = float(T * args.steps * world)
    value = frames_all / (ms / 1000.0)
    feats_per_s = rows_all / (ms / 1000.0)

    # end to end through the public API from pinned host memory
    e2e = None
    if not args.no_e2e:
        try:
            host = torch.empty(video.shape, dtype=torch.uint16, pin_memory=True)
            host.copy_(video)
            host_np = host.numpy()
            e2e_frames = T
        except Exception:
            e2e_frames = min(T, 256)
            host = torch.empty((e2e_frames, S, S), dtype=torch.uint16, pin_memory=True)
            host.copy_(video[:e2e_frames])
            host_np = host.numpy()
        kw = dict(minmass=CONFIG["minmass"], search_range=CONFIG["search_range"], memory=CONFIG["memory"],
                  tqdm=False)
        df = gt.batch(host_np, CONFIG["diameter"], **kw)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d2h = 0
        for _ in range(args.steps):
            df = gt.batch(host_np, CONFIG["diameter"], **kw)
            # float columns travel as float32, integer columns as int64
            d2h += len(df) * sum(8 if df[c].dtype == np.int64 else 4 for c in df.columns)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": e2e_frames * args.steps * world / e2e_s, "unit": "frames/s",
               "h2d_bytes_per_step": int(host_np.nbytes), "d2h_bytes_per_step": int(d2h // args.steps),
               "frames_per_step": e2e_frames}
        del host

    # roofline of the dominant kernel
    peak, peak_kind = load_peaks()
    total_k = sum(v[1] for v in kernels.values()) or 1.0
    # the bandpass + local-max kernel: the longest kernel on the locate stream,
    # whose input read is the step's algorithmic traffic (the linker's kernels
    # run on their own stream beside it)
    dom = ("bandpass_localmax", kernels["bandpass_localmax"]) if "bandpass_localmax" in kernels else (
        max(kernels.items(), key=lambda kv: kv[1][1]) if kernels else ("bandpass_localmax", (1, 1.0)))
    feats_per_frame = rows_all / frames_all
    bytes_per_frame = S * S * 2 + feats_per_frame * 48.0
    # frames per launch of the per-chunk kernels: the engine's chunk size
    frames_per_launch = (T * args.steps) / max(1, kernels.get(dom[0], (1, 1))[0])
    achieved = None
    if dom[1][1] > 0:
        avg_launch_s = dom[1][1] / 1000.0 / dom[1][0]
        achieved = bytes_per_frame * frames_per_launch / avg_launch_s / 1e9
    traffic = load_traffic().get(dom[0])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": (traffic["dram_bytes_per_frame"] * frames_per_launch) if traffic else None,
                "kernel": dom[0], "peak_kind": peak_kind,
                "algorithmic_bytes_per_frame": bytes_per_frame,
                "kernel_share": {k: round(v[1] / total_k, 4) for k, v in kernels.items()},
                "whole_step_frac": frames_all * bytes_per_frame / (ms / 1000.0) / 1e9 / peak}
    # the kernel is bound by instruction issue, not HBM: its thread-instructions
    # per pixel (ncu) against the per-pixel operation floor, and the issue rate
    # it reaches against the SMs' peak (148 SMs x 4 schedulers x 32 lanes per clock)
    issue = load_issue().get(dom[0])
    issue_roofline = None
    if issue and dom[1][1] > 0:
        sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
        avg_launch_s = dom[1][1] / 1000.0 / dom[1][0]
        tipx = float(issue["thread_instr_per_px"])
        achieved_i = tipx * S * S * frames_per_launch / avg_launch_s / 1e12
        peak_i = 148 * 4 * 32 * sm_mhz * 1e6 / 1e12
        issue_roofline = {"unit": "T thread-instr/s", "thread_instr_per_px": tipx,
                          "floor_instr_per_px": issue.get("floor_instr_per_px"),
                          "floor": issue.get("floor"), "achieved": achieved_i, "peak": peak_i,
                          "frac": achieved_i / peak_i, "fp32_lane_ops_per_px": issue.get("fp32_lane_ops_per_px"),
                          "us_per_frame": avg_launch_s / frames_per_launch * 1e6, "source": issue.get("source")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = os.cpu_count() or 1
        n = args.cpu_sample or cpu_sample_frames(cores, T)
        sample = video[:n].cpu().numpy()
        fps, dt, _ = cpu_baseline(sample, p, cores)
        cpu = {"value": fps, "unit": "frames/s", "cores": cores, "kind": "port",
               "sample": "first %d frames of the workload (%.1f s of CPU work)" % (n, dt)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(CONFIG, frames=T, height=S, width=S,
                               parallelism="dp%d (one video per rank)" % world),
                "features_per_s": feats_per_s, "features_per_frame": feats_per_frame,
                "candidates_per_frame": cands_per_frame,
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "issue_roofline": issue_roofline,
                "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
