"""Autotuner of the render launch (no counterpart in the reference, whose
renderer runs a fixed rayon row loop, renderer.rs:684).

The knobs are rt_set_tuning's: the path-pool capacity (how many paths are in
flight; memory, and how long the final drain runs on a partial wavefront),
the grids of the persistent traversal kernels and of the shading kernels, and
the node layout the traversal reads: the reference's 224-byte 8-wide float
nodes, their 8-bit quantised 128-byte copy, or 4-wide 112-byte nodes over the
same binary tree — the BVH width the reference picks by target
(bvh.rs:10-14).
Every path draws its random numbers from (pixel, sample), so the knobs change
speed and memory, never the image.  The tuner times each candidate on a short
render of the frame it will serve (a probe of at most PROBE_SAMPLES path
samples), keeps the fastest, sets it on the scene and caches it under the
caller's key.  A layout the scene lacks (a quantised copy beyond its range,
4-wide nodes of a tree built on the host) is skipped.
"""
import ctypes as C
import itertools
import math

from . import abi

SPACE = {"max_paths": (1 << 21, 1 << 22, 1 << 23), "trace_blocks_per_sm": (4, 6), "shade_blocks_per_sm": (4, 8, 16),
         "node_format": (abi.RT_NODES_FULL, abi.RT_NODES_QUANTISED, abi.RT_NODES_WIDE4)}
PROBE_SAMPLES = 1 << 24
_cache = {}


def candidates(space=None):
    """Every combination of the space's values, as rt_set_tuning keyword dicts."""
    space = space or SPACE
    keys = sorted(space)
    return [dict(zip(keys, vals)) for vals in itertools.product(*(space[k] for k in keys))]


def probe_params(params, probe_samples=PROBE_SAMPLES):
    """The frame's pass parameters with as many samples per pixel as fit the probe budget."""
    q = abi.RtPassParams()
    C.pointer(q)[0] = params
    npix = max(1, q.width * q.height)
    q.n_samples = max(1, min(q.n_samples, math.ceil(probe_samples / npix)))
    return q


def autotune(gs, cam, params, key=None, space=None, repeats=2, timer=None):
    """Time every candidate tuning, set the fastest on `gs` and return
    (tuning, table of (ms, tuning)).  timer(tuning) -> ms overrides the probe
    render (the default renders probe_params(params) and reads the library's
    CUDA-event time); the best of `repeats` runs counts, so a first run that
    grows the path buffers does not decide.  A cached key skips the timing."""
    if key is not None and key in _cache:
        gs.set_tuning(**_cache[key])
        return _cache[key], None
    if timer is None:
        probe = probe_params(params)

        def timer(t):
            gs.set_tuning(**t)
            gs.render_accumulate(cam, probe)
            return gs.last_stats()["ms"]
    from .renderer import RtError
    table = []
    for t in candidates(space):
        try:
            table.append((min(timer(t) for _ in range(max(1, repeats))), t))
        except RtError:
            continue                    # a layout this scene does not have
    best = min(table, key=lambda x: x[0])[1]
    gs.set_tuning(**best)
    if key is not None:
        _cache[key] = best
    return best, table


def clear_cache():
    _cache.clear()
