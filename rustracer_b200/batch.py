"""Batched rendering: many independent frames of several scenes on one GPU.

`run_packed` is the batch service: the requests of each scene kind go into
one packed rt_render_batch call — one wavefront pool draws samples from all
of them, passes of a few samples per pixel of every unfinished request — and
the scene kinds' calls run concurrently, each on its handle's stream.  A
request's latency is the start of its call plus the device time at which the
pass that finished it ended.

`run_batch` is the frame-at-a-time service it replaces: worker threads with
their own handles take jobs from one queue and render each alone
(rt_render_accumulate); with one worker it is the sequential baseline.  Both
report the aggregate path-sample rate and the per-request latencies from the
batch's start.
"""
import math
import queue
import threading
import time

import numpy as np

from . import configs
from .renderer import GpuScene, pass_params
from .scene import make_camera

SCENES = ("box", "icosphere", "gem")


def make_jobs(seed=0, n=64, scenes=SCENES, min_width=128, max_width=1920, min_spp=4, max_spp=256):
    """The batch workload: scene uniform over `scenes`, width log-uniform in
    [min_width, max_width], aspect 1:1 / 4:3 / 16:9, spp log-uniform in
    [min_spp, max_spp], camera orbiting the scene (azimuth U[0, 360), elevation U[10, 40])."""
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(n):
        scene = scenes[int(rng.integers(len(scenes)))]
        w = int(round(math.exp(rng.uniform(math.log(min_width), math.log(max_width)))))
        aspect = (1.0, 4.0 / 3.0, 16.0 / 9.0)[int(rng.integers(3))]
        h = max(16, int(round(w / aspect)))
        spp = int(round(math.exp(rng.uniform(math.log(min_spp), math.log(max_spp)))))
        jobs.append(dict(id=k, scene=scene, width=w, height=h, spp=spp, azimuth=float(rng.uniform(0.0, 360.0)),
                         elevation=float(rng.uniform(10.0, 40.0)), seed=int(rng.integers(1 << 30))))
    return jobs


_ORBIT = {"box": ((0.5, 0.5, 0.5), 1.9), "icosphere": ((0.0, -0.15, 0.0), 3.7), "gem": ((0.0, 0.35, 0.0), 2.7)}
_DEPTH = {"box": 8, "icosphere": 12, "gem": 32}


def job_camera(job):
    look_at, dist = _ORBIT[job["scene"]]
    az, el = math.radians(job["azimuth"]), math.radians(job["elevation"])
    la = np.asarray(look_at, np.float64)
    lf = la + dist * np.array([math.cos(el) * math.sin(az), math.sin(el), -math.cos(el) * math.cos(az)])
    return make_camera(tuple(lf), tuple(la), vfov=40.0, aspect=job["width"] / job["height"])


def build_scene(kind):
    if kind == "box":
        return configs.box_scene()[0]
    if kind == "icosphere":
        return configs.icosphere_scene(env_w=1024, env_h=512)[0]
    if kind == "gem":
        return configs.gem_scene(env_w=512, env_h=256)[0]
    raise ValueError(kind)


def render_job(handles, job):
    """One frame into host accumulators (sum, M2, count)."""
    g = handles[job["scene"]]
    p = pass_params(job["width"], job["height"], 0, job["spp"], int(math.sqrt(job["spp"])), _DEPTH[job["scene"]], 4,
                    1.0, job["seed"])
    return g.render_accumulate(job_camera(job), p)


def tune_kinds(handles, jobs):
    """Autotune each scene kind on its largest job (autotune.py) and set the
    result on every handle of that kind; returns {kind: tuning}."""
    from . import autotune
    out = {}
    for k in sorted({j["scene"] for j in jobs}):
        job = max((j for j in jobs if j["scene"] == k), key=lambda j: j["width"] * j["height"] * j["spp"])
        p = pass_params(job["width"], job["height"], 0, job["spp"], int(math.sqrt(job["spp"])), _DEPTH[k], 4, 1.0,
                        job["seed"])
        best, _ = autotune.autotune(handles[0][k], job_camera(job), p)
        for h in handles[1:]:
            h[k].set_tuning(**best)
        out[k] = best
    return out


def run_batch(jobs, workers=4, device=0, builders=None, keep_outputs=False, tune=False):
    """Render `jobs` with `workers` concurrent threads; returns dict with the
    wall time, per-job latencies (s), the tunings when `tune` (autotuned per
    scene kind before the clock starts) and the outputs when asked."""
    builders = builders or {}
    kinds = sorted({j["scene"] for j in jobs})
    descs = {k: builders[k] if k in builders else build_scene(k) for k in kinds}
    handles = [{k: GpuScene(descs[k], device=device) for k in kinds} for _ in range(workers)]
    tunings = tune_kinds(handles, jobs) if tune else None
    for h in handles:                                    # warm the buffers of every handle
        for k in kinds:
            render_job(h, dict(scene=k, width=64, height=64, spp=1, azimuth=0.0, elevation=20.0, seed=0))
    q = queue.Queue()
    for j in jobs:
        q.put(j)
    lat, outs, errors = {}, {}, []
    t0 = time.perf_counter()

    def worker(h):
        while True:
            try:
                j = q.get_nowait()
            except queue.Empty:
                return
            try:
                out = render_job(h, j)
                lat[j["id"]] = time.perf_counter() - t0
                if keep_outputs:
                    outs[j["id"]] = out
            except Exception as e:   # surfaced after the batch
                errors.append(e)

    threads = [threading.Thread(target=worker, args=(h,)) for h in handles]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    if errors:
        raise errors[0]
    samples = sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    ls = np.array([lat[j["id"]] for j in jobs])
    return dict(wall_s=wall, path_samples=samples, rate=samples / wall, p50_s=float(np.percentile(ls, 50)),
                p99_s=float(np.percentile(ls, 99)), latencies=lat, outputs=outs, tunings=tunings)


def batch_request(job):
    """A job of make_jobs as an rt_render_batch request (the samples of render_job)."""
    return dict(cam=job_camera(job), width=job["width"], height=job["height"], spp=job["spp"],
                strata=int(math.sqrt(job["spp"])), sample_idx=0, seed=job["seed"])


def run_packed(jobs, device=0, builders=None, keep_outputs=False, tune=False, window=0, graph=True):
    """Render `jobs` packed: one rt_render_batch call per scene kind, the
    kinds on concurrent threads (each handle its own stream).  With `graph`,
    every pass of a call replays the handle's captured wavefront graph (the
    job table and launch parameters are read from device memory, so one
    capture serves every pass of the same pool size).  Returns the same
    summary as run_batch."""
    builders = builders or {}
    kinds = sorted({j["scene"] for j in jobs})
    handles = {k: GpuScene(builders[k] if k in builders else build_scene(k), device=device) for k in kinds}
    tunings = tune_kinds([handles], jobs) if tune else None
    if graph:
        for h in handles.values():
            h.set_tuning(**{**h.get_tuning(), "graph": 1})
    for k in kinds:
        # warm each handle: a packed request of one pool's worth of samples
        # grows the path buffers to the pool and, with `graph`, captures the
        # wavefront graph the timed passes replay
        side = 1024
        spp = max(1, -(-handles[k].get_tuning()["max_paths"] // (side * side)))
        warm = dict(scene=k, width=side, height=side, azimuth=0.0, elevation=20.0)
        handles[k].render_batch([dict(cam=job_camera(warm), width=side, height=side, spp=spp, seed=0)],
                                pass_params(64, 64, 0, 1, 1, _DEPTH[k], 4, 1.0, 0))
    lat, outs, errors = {}, {}, []
    t0 = time.perf_counter()

    def worker(k):
        mine = [j for j in jobs if j["scene"] == k]
        try:
            start = time.perf_counter() - t0
            res, done = handles[k].render_batch([batch_request(j) for j in mine],
                                                pass_params(64, 64, 0, 1, 1, _DEPTH[k], 4, 1.0, 0), window=window)
            for j, r, d in zip(mine, res, done):
                lat[j["id"]] = start + float(d) / 1000.0
                if keep_outputs:
                    outs[j["id"]] = r
        except Exception as e:   # surfaced after the batch
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in kinds]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t0
    if errors:
        raise errors[0]
    samples = sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    ls = np.array([lat[j["id"]] for j in jobs])
    return dict(wall_s=wall, path_samples=samples, rate=samples / wall, p50_s=float(np.percentile(ls, 50)),
                p99_s=float(np.percentile(ls, 99)), latencies=lat, outputs=outs, tunings=tunings)
