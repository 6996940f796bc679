"""Rendering with the learned proposal, and the relMSE metric that compares it with cosine bounces.

The reference has no path guiding: every diffuse bounce samples the cosine
lobe (renderer.rs:545-571).  Here a frame is rendered the same way, but the
scene's guide network (rt_guide_*) is trained online from the tracer's own
radiance estimates during the first `train_spp` samples per pixel — one
render call per `train_per_call` samples, each followed by Adam steps on the
records that call wrote — and then frozen for the rest.  Every sample, those
of the training calls included, is an unbiased estimate and is accumulated.
"""
import ctypes as C

import numpy as np

from . import abi


def relmse(x, ref, eps=1e-2):
    """Mean over pixels and channels of (x − ref)² / (ref² + ε)."""
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + eps)))


def _pass(params, sample_idx, n):
    q = abi.RtPassParams()
    C.pointer(q)[0] = params
    q.sample_idx = sample_idx
    q.n_samples = n
    return q


def render_plain(gs, cam, params, spp, sample_idx=0):
    """`spp` samples per pixel with cosine bounces: (mean image, GPU ms)."""
    gs.guide_mode(abi.RT_GUIDE_OFF)
    s, _, c = gs.render_accumulate(cam, _pass(params, sample_idx, spp), reset=True)
    return s / np.maximum(c, 1)[..., None], gs.last_stats()["ms"]


def render_guided(gs, cam, params, spp, train_spp=64, train_per_call=8, guide=None, sample_idx=0):
    """`spp` samples per pixel with a fresh guide network trained during the
    first `train_spp` of them.  Returns (mean image, GPU ms of every render
    call — training steps included —, guide statistics)."""
    gs.guide_init(guide)
    gs.guide_mode(abi.RT_GUIDE_TRAIN)
    ms, done, reset = 0.0, 0, True
    s = c = None
    while done < spp:
        if done < train_spp:
            n = min(train_per_call, train_spp - done, spp - done)
        else:
            gs.guide_mode(abi.RT_GUIDE_SAMPLE)
            n = spp - done
        s, _, c = gs.render_accumulate(cam, _pass(params, sample_idx + done, n), reset=reset)
        ms += gs.last_stats()["ms"]
        reset = False
        done += n
    stats = gs.guide_stats()
    gs.guide_mode(abi.RT_GUIDE_OFF)
    return s / np.maximum(c, 1)[..., None], ms, stats
