"""Benchmark: path samples/s of the render hot path on the icosphere workload.

Workload (one "step"): a complete render of the 1,310,720-triangle displaced
icosphere scene (GGX conductor, diffuse floor, 2048×1024 env map with alias
sampling) at 1920×1080, 64 spp, max depth 12, 4 hero wavelengths — 132,710,400
path samples — accumulated on the device (rt_render_accumulate).  Inputs are
seeded synthetic data (no data set exists for this workload).

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

value    : path samples/s with the scene resident in HBM, device time of each
           step from CUDA events on the library's launching stream, max over
           ranks; every rank renders its own 64 spp (sample indices offset by
           rank) → weak scaling, no collective on the data path.
e2e      : the same metric through the C ABI with HOST output buffers (the
           accumulated image is read back every step), wall time per step.
roofline : the closest-hit traversal kernel (extend).  Algorithmic bytes per
           launch = Σ over that launch's rays of 224 B × 8-wide nodes visited
           + 36 B × triangle tests + 16 B × sphere tests + 64 B × quad tests, as
           counted by the CPU oracle's restatement of the reference traversal
           on rays captured from the GPU's own queues (a subsample per bounce,
           scaled by the bounce's ray count); divided by the kernel's CUDA-event
           time; peak = measured HBM copy bandwidth.
cpu_baseline: the CPU oracle (restatement of the reference's CPU path) on a
           bounded sample of the same frame (bands of 32 rows, 1 spp each,
           ~12 s on all host cores).
secondary: on one GPU the same line carries the box workload (256x256,
           16 spp, depth 8) and the gem workload (57-facet brilliant, 2M-photon
           caustic map rebuilt every step, 1280x720, 256 spp, depth 32), each
           with its value, e2e, roofline and cpu_baseline.
--impl reference: the CPU oracle on all host cores, each step 320 bands of
           32 rows x 1920 px x 1 spp of the icosphere frame (the cpu_baseline
           sampler, ~2.5 s per step), so the default 5 steps time ≥ 10 s.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SPP = 64
W, H = 1920, 1080
DEPTH = 12
HERO = 4
METRIC = "path samples/s (1920x1080 icosphere workload)"
UNIT = "path samples/s"
REF_BANDS = 320         # bands of 32 rows per reference-arm step (~2.5 s on 16 cores: 5 steps ≥ 10 s)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-roofline", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="leave out the box and gem lines")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--mode", choices=["bench", "pass"], default="bench",
                    help="pass: one warm-up call + one measured 16-spp call of the workload, no JSON (profiler driver)")
    ap.add_argument("--config", choices=["icosphere", "gem", "box", "room", "batch", "guided"], default="icosphere",
                    help="gem: the 1280x720 gem workload with its caustic photon map; box: the 256x256 box "
                         "workload (the secondary line's, alone); room: the reference's "
                         "--bench room (1200x800, 128 spp); batch: 64 jobs of the box/icosphere/gem scenes on 4 "
                         "concurrent handles vs one; guided: equal-time relMSE of the learned proposal against "
                         "cosine bounces on the slit-light room (secondary lines; the headline is the icosphere "
                         "workload)")
    ap.add_argument("--ref-spp", type=int, default=16384, help="guided: samples per pixel of the plain reference")
    ap.add_argument("--plain-spp", type=int, default=256, help="guided: samples per pixel of the plain render")
    ap.add_argument("--guide-spp-per-call", type=int, default=8, help="guided: samples per training render call")
    ap.add_argument("--guide-steps", type=int, default=8, help="guided: Adam steps after each training call")
    ap.add_argument("--guide-train-spp", type=int, default=64, help="guided: samples per pixel of training")
    ap.add_argument("--pass-size", default=None, help="pass mode: frame WxH (default: the workload's)")
    ap.add_argument("--pass-spp", type=int, default=None, help="pass mode: samples per pixel of the measured call")
    ap.add_argument("--no-autotune", action="store_true",
                    help="icosphere: keep the built-in launch grids instead of autotune.py's choice")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ── clocks during the timed region ───────────────────────────────────────────
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i - 5] for r in self.rows for i in range(5, 9) if r[i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ── CPU legs (the oracle is the checker and the CPU baseline, never the product) ──
def cpu_band_rate(sb, st, seconds, threads):
    """Oracle samples/s on bands of 32 rows × full width × 1 spp until `seconds` pass."""
    from oracle import oracle as O
    from rustracer_b200.renderer import pass_params
    o = O.OracleScene(sb)
    n = 0
    t0 = time.perf_counter()
    k = 0
    while True:
        row0 = (k * 97) % (H - 32)
        p = pass_params(W, H, k, 1, int(np.sqrt(SPP)), DEPTH, HERO, 1.0, 1000 + k)
        o.render_pass(st["camera"], p, threads=threads, rows=(row0, row0 + 32))
        n += 32 * W
        k += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            return n / el, f"{k} bands of 32 rows x {W} px x 1 spp ({n} path samples, {el:.1f} s)"


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from rustracer_b200 import configs
    sb, st = configs.icosphere_scene(seed=2)
    threads = os.cpu_count() or 1
    from oracle import oracle as O
    from rustracer_b200.renderer import pass_params
    o = O.OracleScene(sb)

    def band(k):
        row0 = (k * 97) % (H - 32)
        p = pass_params(W, H, k, 1, int(np.sqrt(SPP)), DEPTH, HERO, 1.0, 1000 + k)
        o.render_pass(st["camera"], p, threads=threads, rows=(row0, row0 + 32))
        return 32 * W

    def step(k, bands=REF_BANDS):
        return sum(band(k * REF_BANDS + b) for b in range(bands))

    for k in range(args.warmup):
        step(k, REF_BANDS // 8)                 # warm-up steps at an eighth of the size
    t0 = time.perf_counter()
    n = sum(step(args.warmup + k) for k in range(args.steps))
    el = time.perf_counter() - t0
    v = n / el
    sample = (f"{args.steps} steps of {REF_BANDS} bands of 32 rows x {W} px x 1 spp of the {W}x{H} frame "
              f"({n} path samples, {el:.1f} s)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el * 1000 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": "icosphere8 1310720 tris 1920x1080 depth12 hero4 (CPU oracle: restatement of the "
                               "reference's CPU path; the Rust reference cannot be built here)",
                   "parallelism": f"{threads} host threads"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_ours(args):
    import torch
    import ctypes as C
    from rustracer_b200 import abi, configs
    from rustracer_b200.renderer import GpuScene, pass_params

    ws, rank, local = dist_env()
    if ws != args.gpus:
        sys.exit(f"bench.py --gpus {args.gpus} runs one process per GPU: start it with "
                 f"`python -m torch.distributed.run --nproc-per-node {args.gpus} ... bench.py --gpus {args.gpus}` "
                 f"(WORLD_SIZE is {ws})")
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    sb, st = configs.icosphere_scene(seed=2)
    scene = GpuScene(sb, device=local)
    cam = st["camera"]
    per_step = W * H * SPP

    def params(step):
        return pass_params(W, H, (rank * 100003 + step) * SPP, SPP, int(np.sqrt(SPP)), DEPTH, HERO, 1.0, 2)

    tuning = None
    if not args.no_autotune:
        # the library's launch autotuner on a probe of this frame, before any timing
        # (every rank tunes its own GPU; the image does not depend on the choice)
        from rustracer_b200 import autotune
        tuning, _ = autotune.autotune(scene, cam, params(1000))

    outs = (torch.zeros((H, W, 3), device=dev), torch.zeros((H, W, 3), device=dev),
            torch.zeros((H, W), dtype=torch.int32, device=dev))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)   # 256 MB > 126 MB L2

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    for k in range(args.warmup):
        scene.render_accumulate(cam, params(k), outputs=outs)
    flush.fill_(1)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    dev_ms = []
    ext = sh = launches = 0
    barrier()
    torch.cuda.synchronize()
    merge_ms = 0.0
    for k in range(args.steps):
        scene.render_accumulate(cam, params(args.warmup + k), outputs=outs)
        stt = scene.last_stats()
        dev_ms.append(stt["ms"])
        if ws > 1:
            # one frame across the ranks: combine the accumulators (sum, M2, count)
            from rustracer_b200.multigpu import merge_accumulators
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            merge_accumulators(*outs)
            e1.record()
            e1.synchronize()
            dev_ms[-1] += e0.elapsed_time(e1)
            merge_ms += e0.elapsed_time(e1)
        ext += stt["ext_rays"]
        sh += stt["shadow_rays"]
        launches += stt["launches"]
        flush.fill_(k & 0xFF)    # evict L2 between timed steps (not inside the timed region)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    total_ms = sum(dev_ms)
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = ws * per_step * args.steps / (total_ms / 1000.0)

    # e2e: the public C ABI with host output buffers (accumulated image read back every step)
    host = (torch.empty((H, W, 3), pin_memory=True), torch.empty((H, W, 3), pin_memory=True),
            torch.empty((H, W), dtype=torch.int32, pin_memory=True))
    e2e_s = []
    barrier()
    for k in range(max(2, min(args.steps, 3))):
        t0 = time.perf_counter()
        scene.render_accumulate(cam, params(1000 + k), outputs=host)
        e2e_s.append(time.perf_counter() - t0)
    e2e_total = sum(e2e_s)
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_total], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = ws * per_step * len(e2e_s) / e2e_total
    h2d = C.sizeof(abi.RtCamera) + C.sizeof(abi.RtPassParams)
    d2h = H * W * (3 + 3) * 4 + H * W * 4

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded icosphere, Perlin displacement, procedural sky)",
        "config": {"workload": "icosphere8 1310720 tris, GGX conductor + diffuse floor, 2048x1024 env, "
                               "1920x1080, 64 spp, depth 12, hero 4",
                   "spp_per_step": SPP, "path_samples_per_step_per_gpu": per_step,
                   "launch_tuning": tuning or "built-in",
                   "parallelism": f"weak: {ws} rank(s), each its own 64 spp"
                                  + (", accumulators all-reduced every frame (NCCL)" if ws > 1 else ""),
                   "l2": "256 MB buffer written between timed steps; scene (~230 MB) exceeds L2",
                   "bvh_build_ms": scene.build_time_ms()},
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "merge_ms_per_step": merge_ms / args.steps if ws > 1 else None,
        "gpu_launches": int(launches),
        "rays": {"extension": int(ext), "shadow": int(sh),
                 "rays_per_s": (ext + sh) / (sum(dev_ms) / 1000.0)},
    }

    if rank == 0 and not args.no_roofline:
        line["roofline"] = roofline(scene, sb, cam)
    if rank == 0 and not args.no_cpu_baseline and ws == 1:
        threads = os.cpu_count() or 1
        v, sample = cpu_band_rate(sb, st, args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}
    if rank == 0 and ws == 1 and not args.no_secondary:
        # configs 1 and 3 beside the headline (one GPU; the scaling run measures the headline)
        scene.close()
        del outs, flush
        torch.cuda.empty_cache()
        line["secondary"] = [secondary(k, args) for k in ("box", "gem")]
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def roofline(scene, sb, cam, w=W, h=H, spp=SPP, depth=DEPTH, hero=HERO, seed=2, traffic_file="extend_icosphere_traffic.txt"):
    """Roofline of the extend (closest-hit) kernel; see the module docstring.
    The kernel is not HBM-bound: its node and primitive fetches are served
    mostly by L1 and L2, so `frac` (algorithmic bytes per second over the HBM
    copy peak) measures how fast the cache hierarchy delivers the reference
    layout's bytes, and `dram_frac` beside it is the DRAM traffic ncu measured
    for the kernel over the same time."""
    from oracle import oracle as O
    from rustracer_b200.renderer import pass_params
    peak, peak_kind = measured_peak()
    strata = int(np.sqrt(np.float32(spp)))
    p1 = pass_params(w, h, 5000, 1, strata, depth, hero, 1.0, seed)
    scene.set_profiling(True)
    p = pass_params(w, h, 6000, spp, strata, depth, hero, 1.0, seed)
    scene.render_accumulate(cam, p)
    kt = scene.kernel_times()
    ext_rays = scene.last_stats()["ext_rays"]
    scene.set_profiling(False)
    o = O.OracleScene(sb)
    rng = np.random.default_rng(0)
    total_bytes_pass = 0.0
    per_depth = []
    for d in range(depth):
        r = scene.capture_rays(cam, p1, d, w * h)
        if len(r) == 0:
            break
        sub = r[rng.choice(len(r), size=min(len(r), 20000), replace=False)]
        stt = o.trace_stats(sub)
        bpr = (224.0 * stt[:, 0] + 36.0 * stt[:, 1] + 16.0 * stt[:, 2] + 64.0 * stt[:, 3]).mean()
        total_bytes_pass += bpr * len(r)
        per_depth.append((d, len(r), float(bpr), float(stt[:, 0].mean()), float(stt[:, 1].mean())))
    ext_ms, ext_launches = kt["extend"]
    # total algorithmic bytes of all extend launches of the render ÷ their total device time
    achieved = total_bytes_pass * spp / (ext_ms / 1000.0) / 1e9 if ext_ms > 0 else None
    # DRAM traffic: ncu's bytes per extension ray on this kernel and scene
    # (a profile summary) times this render's extension rays per launch
    traffic, traffic_source = None, None
    tfile = os.path.join(ROOT, "profiles", traffic_file) if traffic_file else None
    if tfile and os.path.exists(tfile):
        for ln in open(tfile):
            if ln.startswith("traffic_bytes_per_ray:"):
                traffic = float(ln.split(":")[1]) * ext_rays / max(1, ext_launches)
            elif ln.startswith("source:"):
                traffic_source = f"profiles/{traffic_file}: ncu on {ln.split(':', 1)[1].strip()}, per extension ray"
    launch_s = ext_ms / 1000.0 / max(1, ext_launches)
    dram_gbs = traffic / launch_s / 1e9 if (traffic and launch_s > 0) else None
    return {"kernel": "k_extend (8-wide BVH closest hit)", "bound": "hbm",
            "limiter": "L1/TEX throughput and load latency (node fetches hit L1/L2), not DRAM bandwidth",
            "achieved": achieved, "peak": peak,
            "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak if achieved else None,
            "traffic": traffic, "traffic_source": traffic_source, "dram_gbs": dram_gbs,
            "dram_frac": dram_gbs / peak if dram_gbs else None,
            "algorithmic_bytes_per_launch": total_bytes_pass * spp / max(1, ext_launches),
            "launches": ext_launches, "kernel_ms": ext_ms,
            "stage_ms": {k: v[0] for k, v in kt.items()},
            "per_bounce": [{"depth": d, "rays": n, "bytes_per_ray": b, "nodes_per_ray": nn, "tris_per_ray": tt}
                           for d, n, b, nn, tt in per_depth]}


def secondary(kind, args):
    """One secondary workload of the headline line (one GPU): `value` from the
    library's CUDA-event time of each step (plus the photon build's device
    time for the gem), `e2e` through rt_render_accumulate with host output
    buffers (and the photon build) timed by the host clock, the extend
    kernel's roofline and the oracle's CPU rate on bands of the same frame."""
    import torch
    from oracle import oracle as O
    from rustracer_b200 import configs
    from rustracer_b200.renderer import GpuScene, pass_params
    if kind == "box":
        sb, st = configs.box_scene()
        # a frame is ~1.3 ms: at least 400 timed frames (~0.5 s), so the clock
        # sampler (every 200 ms) sees the timed region
        steps, warm = max(args.steps, 400), args.warmup
    else:
        sb, st = configs.gem_scene()
        steps, warm = max(1, min(args.steps, 3)), args.warmup
    w, h, spp, depth, hero = st["width"], st["height"], st["spp"], st["max_depth"], st["hero"]
    strata = int(np.sqrt(np.float32(spp)))
    cam = st["camera"]
    scene = GpuScene(sb, device=0)
    dev = torch.device("cuda", 0)
    outs = (torch.zeros((h, w, 3), device=dev), torch.zeros((h, w, 3), device=dev),
            torch.zeros((h, w), dtype=torch.int32, device=dev))
    host = (torch.empty((h, w, 3), pin_memory=True), torch.empty((h, w, 3), pin_memory=True),
            torch.empty((h, w), dtype=torch.int32, pin_memory=True))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    photons = kind == "gem"
    stored = []

    def step(k, o):
        ph_ms = 0.0
        if photons:
            stored.append(scene.photon_build(st["photon_params"](seed=k)))
            ph_ms = sum(scene.photon_stage_ms())
        scene.render_accumulate(cam, pass_params(w, h, k * spp, spp, strata, depth, hero, 1.0, 7), outputs=o)
        stt = scene.last_stats()
        return stt["ms"] + ph_ms, ph_ms, stt

    tuning = None
    if not args.no_autotune:
        # the library's launch autotuner on a probe of this frame, as for the headline
        from rustracer_b200 import autotune
        if photons:
            scene.photon_build(st["photon_params"](seed=0))
        tuning, _ = autotune.autotune(scene, cam, pass_params(w, h, 0, spp, strata, depth, hero, 1.0, 7))
    for k in range(warm):
        step(k, outs)
    flush.fill_(1)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    ms, ph, ext, sh, launches = [], [], 0, 0, 0
    for k in range(steps):
        a, b, stt = step(warm + k, outs)
        ms.append(a)
        ph.append(b)
        ext += stt["ext_rays"]
        sh += stt["shadow_rays"]
        launches += stt["launches"]
        flush.fill_(k & 0xFF)
    torch.cuda.synchronize()
    clk = clocks.stop()
    per_step = w * h * spp
    e2e_s = []
    for k in range(50 if kind == "box" else max(2, min(steps, 3))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step(1000 + k, host)
        e2e_s.append(time.perf_counter() - t0)
    line = {
        "workload": st["name"], "metric": f"path samples/s ({w}x{h} {kind} workload)",
        "value": per_step * steps / (sum(ms) / 1000.0), "unit": UNIT, "steps": steps, "warmup": warm,
        "ms_per_step": sum(ms) / steps, "clocks": clk, "gpu_launches": int(launches),
        "e2e": {"value": per_step * len(e2e_s) / sum(e2e_s), "unit": UNIT,
                "h2d_bytes_per_step": 136, "d2h_bytes_per_step": h * w * (3 + 3) * 4 + h * w * 4},
        "rays": {"extension": int(ext), "shadow": int(sh), "rays_per_s": (ext + sh) / (sum(ms) / 1000.0)},
        "l2": "256 MB buffer written between timed steps",
        "launch_tuning": tuning or "built-in",
    }
    if photons:
        line["photon_map"] = {"emitted": st["photons"], "stored_mean": int(np.mean(stored)),
                              "build_ms": float(np.mean(ph)),
                              "stage_ms": dict(zip(("trace", "compact", "tree"), scene.photon_stage_ms())),
                              "source": "the two light quads, aimed at the stone's bounding sphere (projection map)",
                              "knn_k": st["knn_k"], "radius_max": st["radius_max"]}
    if not args.no_roofline:
        line["roofline"] = roofline(scene, sb, cam, w, h, min(spp, 16), depth, hero, 7,
                                    traffic_file=f"extend_{kind}_traffic.txt")
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        o = O.OracleScene(sb)
        if photons:
            o.photon_build(st["photon_params"](seed=1))
        n, k, t0 = 0, 0, time.perf_counter()
        while time.perf_counter() - t0 < args.cpu_seconds:
            row0 = (k * 61) % max(1, h - 32)
            o.render_pass(cam, pass_params(w, h, k, 1, strata, depth, hero, 1.0, 900 + k), threads=threads,
                          rows=(row0, min(h, row0 + 32)))
            n += min(32, h) * w
            k += 1
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": n / el, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{k} bands of 32 rows x {w} px x 1 spp ({n} path samples, {el:.1f} s)"
                                          + ("; photon map built once before timing" if photons else "")}
    scene.close()
    del outs, host, flush
    torch.cuda.empty_cache()
    return line


def run_gem(args):
    """Secondary workload: a round brilliant in dispersive diamond with a k-NN
    caustic photon map.  One step = rebuild the photon map (2M photons emitted)
    and render 1280x720 at 256 spp, depth 32, 4 hero wavelengths.  The render is
    timed by the library's CUDA events, the photon build (which synchronises) by
    the host clock around it."""
    import torch
    from rustracer_b200 import configs, photons
    from rustracer_b200.renderer import GpuScene, pass_params
    sb, st = configs.gem_scene()
    w, h, spp = st["width"], st["height"], st["spp"]
    scene = GpuScene(sb, device=0)
    dev = torch.device("cuda", 0)
    outs = (torch.zeros((h, w, 3), device=dev), torch.zeros((h, w, 3), device=dev),
            torch.zeros((h, w), dtype=torch.int32, device=dev))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def step(k):
        pp = photons.caustic_params(sb, st["photons"], st["radius_max"], knn_k=st["knn_k"], seed=k,
                                    env_dir=st["env_dir"], env_color=st["env_color"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n = scene.photon_build(pp)
        t_ph = (time.perf_counter() - t0) * 1000.0
        scene.render_accumulate(st["camera"], pass_params(w, h, k * spp, spp, int(np.sqrt(spp)), st["max_depth"],
                                                          st["hero"], 1.0, 3), outputs=outs)
        stt = scene.last_stats()
        return t_ph, stt["ms"], n, stt

    for k in range(args.warmup):
        step(k)
    flush.fill_(1)
    clocks = ClockSampler(0)
    clocks.start()
    ph_ms, r_ms, stored, ext, sh = [], [], [], 0, 0
    for k in range(args.steps):
        a, b, n, stt = step(args.warmup + k)
        ph_ms.append(a)
        r_ms.append(b)
        stored.append(n)
        ext += stt["ext_rays"]
        sh += stt["shadow_rays"]
        flush.fill_(k & 0xFF)
    torch.cuda.synchronize()
    clk = clocks.stop()
    total = sum(ph_ms) + sum(r_ms)
    per_step = w * h * spp
    line = {
        "metric": "path samples/s (1280x720 gem workload)", "value": per_step * args.steps / (total / 1000.0),
        "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (generated round brilliant, procedural sky at 0.1)",
        "config": {"workload": f"{st['name']}, photon map {st['photons']} emitted, k-NN {st['knn_k']}, "
                               f"r <= {st['radius_max']}",
                   "photon_build_ms": statistics.mean(ph_ms), "render_ms": statistics.mean(r_ms),
                   "photons_stored": int(statistics.mean(stored)),
                   "l2": "256 MB buffer written between timed steps"},
        "clocks": clk,
        "rays": {"extension": int(ext), "shadow": int(sh), "rays_per_s": (ext + sh) / (sum(r_ms) / 1000.0)},
    }
    print(json.dumps(line), flush=True)


def run_room(args):
    """Secondary workload: the reference's own benchmark room (bench.toml's
    layout; --bench renders it at 1200x800, 128 spp, after building the caustic
    photon map once, main.rs:84-117).  One step = 128 spp of the frame on the
    device accumulators, timed by the library's CUDA events; e2e adds the read
    of the developed 8-bit frame.  The CPU baseline is the oracle on bands of
    the same frame at 1 spp."""
    import torch
    from rustracer_b200 import configs, photons
    from rustracer_b200.renderer import GpuScene, pass_params
    from oracle import oracle as O
    sb, st = configs.gem_room_scene()
    w, h, spp, depth = st["width"], st["height"], st["spp"], st["max_depth"]
    strata = int(np.sqrt(np.float32(spp)))
    scene = GpuScene(sb, device=0)
    n_stored = scene.photon_build(photons.caustic_params(sb, st["photons"], st["radius"], seed=1))
    dev = torch.device("cuda", 0)
    outs = (torch.zeros((h, w, 3), device=dev), torch.zeros((h, w, 3), device=dev),
            torch.zeros((h, w), dtype=torch.int32, device=dev))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def step(k, develop=False):
        scene.render_accumulate(st["camera"], pass_params(w, h, k * spp, spp, strata, depth, st["hero"], 1.0, 5),
                                outputs=outs)
        ms = scene.last_stats()["ms"]
        if develop:
            scene.develop(w, h)
        return ms

    for k in range(args.warmup):
        step(k)
    flush.fill_(1)
    clocks = ClockSampler(0)
    clocks.start()
    r_ms, e2e_ms = [], []
    for k in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r_ms.append(step(args.warmup + k, develop=True))
        e2e_ms.append((time.perf_counter() - t0) * 1000.0)
        flush.fill_(k & 0xFF)
    torch.cuda.synchronize()
    clk = clocks.stop()
    per_step = w * h * spp
    line = {
        "metric": "path samples/s (1200x800 gem room, the reference's --bench scene)",
        "value": per_step * args.steps / (sum(r_ms) / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(r_ms), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (bench.toml layout; the 1,400-face OBJ ball replaced by a generated 1,400-face ball)",
        "config": {"workload": f"{st['name']}: 2 analytic gems, PBR gold ball, blackbody panel, dusk sky, "
                               f"{w}x{h}, {spp} spp, depth {depth}, hero 1, photon map {st['photons']} emitted "
                               f"(r {st['radius']}, {n_stored} stored)",
                   "l2": "256 MB buffer written between timed steps"},
        "clocks": clk,
        "e2e": {"value": per_step * args.steps / (sum(e2e_ms) / 1000.0), "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": w * h * 3},
    }
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        o = O.OracleScene(sb)
        o.photon_build(photons.caustic_params(sb, st["photons"], st["radius"], seed=1))
        n, k, t0 = 0, 0, time.perf_counter()
        while time.perf_counter() - t0 < 10.0:
            row0 = (k * 61) % (h - 32)
            o.render_pass(st["camera"], pass_params(w, h, k, 1, strata, depth, st["hero"], 1.0, 900 + k),
                          threads=threads, rows=(row0, row0 + 32))
            n += 32 * w
            k += 1
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": n / el, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{k} bands of 32 rows x {w} px x 1 spp ({n} path samples, {el:.1f} s)"}
    print(json.dumps(line), flush=True)


def run_guided(args):
    """Learned proposal against cosine bounces at equal GPU time on the
    slit-light room (1280x720, depth 24): a plain render of --plain-spp is
    timed and scored against a plain --ref-spp reference; a fresh network is
    trained during the guided render's first 64 spp (render calls of 8 spp,
    8 Adam steps of 65,536 records after each) and then frozen, and the
    guided render's relMSE is read at checkpoints.  `value` is the GPU time
    the guided render needs to reach the plain render's relMSE over the plain
    render's time (log-log interpolation between checkpoints; training
    included), lower is better.  Times are the library's CUDA-event times of
    the render calls; accumulators stay on the device."""
    import torch
    from rustracer_b200 import abi, configs
    from rustracer_b200.guiding import relmse
    from rustracer_b200.renderer import GpuScene, guide_params, pass_params
    sb, st = configs.guided_box_scene()
    w, h, depth, hero = st["width"], st["height"], st["max_depth"], st["hero"]
    scene = GpuScene(sb, device=0)
    cam = st["camera"]
    dev = torch.device("cuda", 0)
    outs = (torch.zeros((h, w, 3), device=dev), torch.zeros((h, w, 3), device=dev),
            torch.zeros((h, w), dtype=torch.int32, device=dev))

    def acc(sample_idx, n, seed, reset):
        scene.render_accumulate(cam, pass_params(w, h, sample_idx, n, 16, depth, hero, 1.0, seed), reset=reset,
                                outputs=outs)
        return scene.last_stats()["ms"]

    def image():
        s, _, c = outs
        return (s / c.clamp(min=1)[..., None].float()).cpu().numpy()

    ref_ms = 0.0
    for k in range(0, args.ref_spp, 512):
        ref_ms += acc(k, min(512, args.ref_spp - k), 101, k == 0)
    ref = image()
    scene.guide_mode(abi.RT_GUIDE_OFF)
    acc(0, 4, 7, True)                                    # warm-up
    t_p = acc(0, args.plain_spp, 7, True)
    e_p = relmse(image(), ref)
    scene.guide_init(guide_params(batch=65536, steps_per_pass=args.guide_steps, seed=3))
    scene.guide_mode(abi.RT_GUIDE_TRAIN)
    t_g, done, pts = 0.0, 0, []
    while done < args.guide_train_spp:
        t_g += acc(done, args.guide_spp_per_call, 9, done == 0)
        done += args.guide_spp_per_call
    pts.append((t_g, relmse(image(), ref), done))
    scene.guide_mode(abi.RT_GUIDE_SAMPLE)
    while done < 4 * args.plain_spp and (pts[-1][1] > e_p or t_g < t_p):
        n = max(16, done // 4)
        t_g += acc(done, n, 9, False)
        done += n
        pts.append((t_g, relmse(image(), ref), done))
    gstats = scene.guide_stats()
    scene.guide_mode(abi.RT_GUIDE_OFF)
    t_plain_frozen = acc(0, 64, 13, True)
    scene.guide_mode(abi.RT_GUIDE_SAMPLE)
    t_guided_frozen = acc(0, 64, 13, True)
    scene.guide_mode(abi.RT_GUIDE_OFF)

    def interp(ki, kv, x):
        # log-log interpolation of column kv where column ki = x
        for a, b in zip(pts, pts[1:]):
            if (a[ki] - x) * (b[ki] - x) <= 0 and a[ki] != b[ki]:
                f = (np.log(x) - np.log(a[ki])) / (np.log(b[ki]) - np.log(a[ki]))
                return float(np.exp(np.log(a[kv]) + f * (np.log(b[kv]) - np.log(a[kv]))))
        return None
    t_match = interp(1, 0, e_p) if pts[-1][1] <= e_p else None
    line = {
        "metric": "equal-time relMSE: guided GPU time to reach the plain render's relMSE / plain GPU time "
                  "(slit-light room)",
        "value": (t_match / t_p) if t_match else None, "unit": "x", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": t_p, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16",
        "data": "synthetic (box room, slit light, round brilliant, Perlin medium; random-init network trained online)",
        "config": {"workload": st["name"], "reference": f"plain {args.ref_spp} spp ({ref_ms / 1000:.1f} s)",
                   "plain": f"{args.plain_spp} spp, {t_p:.0f} ms, relMSE {e_p:.5g}",
                   "guided_relmse_at_equal_time": interp(0, 1, t_p),
                   "guided_checkpoints": [{"ms": round(a, 1), "relmse": b, "spp": c} for a, b, c in pts],
                   "cost_per_spp_ms": {"plain": round(t_plain_frozen / 64, 3), "guided": round(t_guided_frozen / 64, 3)},
                   "training": {"spp": args.guide_train_spp, "spp_per_call": args.guide_spp_per_call,
                                "steps_per_call": args.guide_steps,
                                "records": gstats["records"], "samples": gstats["samples"],
                                "adam_steps": gstats["steps"], "train_ms": round(gstats["train_ms"], 1)},
                   "relmse": "mean over pixels and channels of (x - ref)^2 / (ref^2 + 1e-2)"},
    }
    print(json.dumps(line), flush=True)


def run_batch(args):
    """Secondary workload: 64 requests (scene, size, aspect, spp and camera
    orbit drawn from a seed).  Packed: each scene kind's requests in one
    rt_render_batch call (one wavefront pool over all of them), every pass a
    replay of the kind's captured wavefront graph, the kinds on concurrent
    streams, launch tuning per kind by the autotuner; one untimed batch first.
    Beside it: the same packed calls on the host-driven loop.  Baselines:
    the same requests one frame at a time on 4 concurrent handles, and
    sequentially on one.  Wall clock from submission to the last frame;
    per-request latency from submission to that request's completion."""
    from rustracer_b200 import batch
    jobs = batch.make_jobs(seed=0, n=64)
    builders = {k: batch.build_scene(k) for k in batch.SCENES}
    batch.run_packed(jobs, builders=builders, tune=True)          # untimed warm-up step
    packed = batch.run_packed(jobs, builders=builders, tune=True)
    loop = batch.run_packed(jobs, builders=builders, tune=True, graph=False)
    conc = batch.run_batch(jobs, workers=4, builders=builders)
    seq = batch.run_batch(jobs, workers=1, builders=builders)
    line = {
        "metric": "path samples/s (64-request batch)", "value": packed["rate"], "unit": UNIT, "n_gpus": 1, "steps": 1,
        "warmup": 1, "ms_per_step": packed["wall_s"] * 1000.0, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (box, icosphere, gem scenes; seeded request list)",
        "config": {"workload": "64 requests: scene in {box, icosphere, gem}, width log-U[128,1920], aspect "
                               "{1:1, 4:3, 16:9}, spp log-U[4,256], orbiting camera",
                   "path_samples": packed["path_samples"],
                   "packing": "one rt_render_batch call per scene kind, 3 concurrent streams, autotuned per kind, "
                              "every pass a replay of the kind's captured wavefront graph"},
        "latency_s": {"p50": packed["p50_s"], "p99": packed["p99_s"]},
        "tunings": packed["tunings"],
        "packed_host_loop": {"value": loop["rate"], "wall_s": loop["wall_s"], "p50": loop["p50_s"], "p99": loop["p99_s"],
                             "note": "the same packed calls with the host queueing each iteration instead of "
                                     "replaying the graph"},
        "frame_at_a_time_4_handles": {"value": conc["rate"], "wall_s": conc["wall_s"], "p50": conc["p50_s"],
                                      "p99": conc["p99_s"]},
        "sequential": {"value": seq["rate"], "wall_s": seq["wall_s"], "p50": seq["p50_s"], "p99": seq["p99_s"]},
        "timing": "host wall clock around the whole batch (the frames run on several streams)",
    }
    print(json.dumps(line), flush=True)


def one_pass(args):
    """Profiler driver: one warm-up call and one measured call of the 1920×1080
    icosphere workload (or --pass-size / --pass-spp), 16 samples per pixel per
    call: 33.2M path samples through the 8.4M-path pool, so most launches run
    on a full, refilled pool as in the timed 64-spp render."""
    import torch
    from rustracer_b200 import configs
    from rustracer_b200.renderer import GpuScene, pass_params
    sb, st = configs.icosphere_scene(seed=2)
    scene = GpuScene(sb, device=0)
    w, h, spp = pass_frame(args, W, H, 16)
    out = torch.zeros((spp, h, w, 3), device="cuda")
    for k in range(2):
        scene.render_pass(st["camera"], pass_params(w, h, spp * k, spp, int(np.sqrt(SPP)), DEPTH, HERO, 1.0, 2), out=out)
        print(f"call {k + 1}", scene.last_stats(), flush=True)
    torch.cuda.synchronize()
    print("pass ok", flush=True)


def pass_frame(args, w, h, spp):
    """The pass mode's frame and samples: the workload's unless --pass-size / --pass-spp."""
    if args.pass_size:
        w, h = (int(x) for x in args.pass_size.lower().split("x"))
    return w, h, args.pass_spp or spp


def one_pass_scene(kind, args):
    """Profiler driver for the box and gem workloads (at their stated frames
    unless --pass-size / --pass-spp): the gem builds its 2M-photon map, then
    one 1-spp warm-up call and one measured 4-spp call (gem) or 16-spp call
    (box) of rt_render_accumulate."""
    from rustracer_b200 import configs
    from rustracer_b200.renderer import GpuScene, pass_params
    sb, st = configs.gem_scene() if kind == "gem" else configs.box_scene()
    depth, hero = st["max_depth"], st["hero"]
    w, h, spp = pass_frame(args, st["width"], st["height"], 4 if kind == "gem" else st["spp"])
    scene = GpuScene(sb, device=0)
    if kind == "gem":
        scene.photon_build(st["photon_params"](seed=1))
    scene.render_accumulate(st["camera"], pass_params(w, h, 0, 1, 1, depth, hero, 1.0, 3))
    print("call 1", scene.last_stats(), flush=True)
    scene.render_accumulate(st["camera"], pass_params(w, h, 1, spp, int(np.sqrt(spp)), depth, hero, 1.0, 3))
    print("call 2", scene.last_stats(), flush=True)
    print("pass ok", flush=True)


def one_pass_guided():
    """Profiler driver for the learned proposal: the 1280×720 slit-light room,
    16 spp of training (4 render calls of 4 spp, 16 Adam steps after each),
    then one frozen guided call of 16 spp."""
    from rustracer_b200 import abi, configs
    from rustracer_b200.renderer import GpuScene, guide_params, pass_params
    sb, st = configs.guided_box_scene()
    w, h, depth, hero = st["width"], st["height"], st["max_depth"], st["hero"]
    scene = GpuScene(sb, device=0)
    scene.guide_init(guide_params(steps_per_pass=16, seed=3))
    scene.guide_mode(abi.RT_GUIDE_TRAIN)
    for k in range(4):
        scene.render_accumulate(st["camera"], pass_params(w, h, 4 * k, 4, 16, depth, hero, 1.0, 9), reset=k == 0)
    scene.guide_mode(abi.RT_GUIDE_SAMPLE)
    scene.render_accumulate(st["camera"], pass_params(w, h, 16, 16, 16, depth, hero, 1.0, 9), reset=False)
    print("pass ok", scene.last_stats(), scene.guide_stats(), flush=True)


def main():
    args = parse()
    if args.mode == "pass":
        if args.config == "guided":
            one_pass_guided()
        elif args.config in ("gem", "box"):
            one_pass_scene(args.config, args)
        else:
            one_pass(args)
        return
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "gem":
        run_gem(args)
    elif args.config == "box":
        print(json.dumps(secondary("box", args)), flush=True)
    elif args.config == "room":
        run_room(args)
    elif args.config == "batch":
        run_batch(args)
    elif args.config == "guided":
        run_guided(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
