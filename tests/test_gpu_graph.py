"""The wavefront as one CUDA graph (RtTuning.graph) and the asynchronous
accumulate entry point (rt_render_accumulate_async + rt_sync).

A graph call runs the same kernels on the same buffers as the host-driven
loop — the pool's first fill, then one conditional node per iteration that
runs while rays remain — so its images are bit-identical.  The graph is
captured on the first call and replayed by later ones with new cameras,
sample indices and seeds (the launch parameters live in device memory); a
changed photon map or tuning makes a new one.  The iteration bound is
checked on the device and reported as RT_ERR_TIMEOUT."""
import numpy as np
import pytest

from rustracer_b200 import configs
from rustracer_b200.renderer import GpuScene, RtError, pass_params

pytestmark = pytest.mark.gpu

RT_ERR_TIMEOUT = 3


def _same(a, b):
    assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.mark.parametrize("name", ["box", "icosphere", "media_box"])
def test_graph_renders_are_bit_identical(name):
    if name == "icosphere":
        sb, st = configs.icosphere_scene(width=128, height=72, levels=5, env_w=512, env_h=256)
    else:
        sb, st = getattr(configs, f"{name}_scene")(width=96, height=64)
    g = GpuScene(sb)
    w, h = 96, 64
    ref = [g.render_pass(st["camera"], pass_params(w, h, 8 * k, 8, 2, st["max_depth"], st["hero"], 1.0, 3 + k))
           for k in range(3)]
    g.set_tuning(graph=1)
    assert g.get_tuning()["graph"] == 1
    # the first call captures the graph, the next two replay it with other
    # sample indices and seeds
    for k in range(3):
        got = g.render_pass(st["camera"], pass_params(w, h, 8 * k, 8, 2, st["max_depth"], st["hero"], 1.0, 3 + k))
        _same(got, ref[k])
    a = g.render_accumulate(st["camera"], pass_params(w, h, 0, 16, 4, st["max_depth"], st["hero"], 1.0, 5))
    g.set_tuning()
    b = g.render_accumulate(st["camera"], pass_params(w, h, 0, 16, 4, st["max_depth"], st["hero"], 1.0, 5))
    for x, y in zip(a, b):
        _same(x, y)


def test_graph_follows_photon_map_rebuilds():
    """The gem with its caustic map: a rebuilt map (another photon count) makes
    a new graph, and every frame equals the host-driven loop's."""
    sb, st = configs.gem_scene(width=96, height=54)
    g = GpuScene(sb)
    p = pass_params(96, 54, 0, 8, 2, st["max_depth"], st["hero"], 1.0, 41)
    refs = []
    for seed in (1, 2):
        g.photon_build(st["photon_params"](seed=seed, n=200_000))
        refs.append(g.render_pass(st["camera"], p))
    g.set_tuning(graph=1)
    for seed, ref in zip((1, 2), refs):
        g.photon_build(st["photon_params"](seed=seed, n=200_000))
        _same(g.render_pass(st["camera"], p), ref)


def test_graph_iteration_bound_returns_timeout():
    sb, st = configs.box_scene(width=64, height=64)
    g = GpuScene(sb)
    p = pass_params(64, 64, 0, 2, 1, 8, 4, 1.0, 9)
    ref = g.render_pass(st["camera"], p)
    g.set_tuning(graph=1, max_iterations=2)
    with pytest.raises(RtError) as e:
        g.render_pass(st["camera"], p)
    assert e.value.code == RT_ERR_TIMEOUT and "iteration bound" in str(e.value)
    g.set_tuning(graph=1)
    _same(g.render_pass(st["camera"], p), ref)


def test_async_accumulate_matches_the_synchronous_call():
    import torch
    sb, st = configs.box_scene(width=128, height=96)
    g = GpuScene(sb)
    p = pass_params(128, 96, 0, 16, 4, 8, 4, 1.0, 7)
    ref = g.render_accumulate(st["camera"], p)
    dev = torch.device("cuda", 0)
    outs = (torch.zeros((96, 128, 3), device=dev), torch.zeros((96, 128, 3), device=dev),
            torch.zeros((96, 128), dtype=torch.int32, device=dev))
    side = torch.cuda.Stream(dev)
    with torch.cuda.stream(side):
        g.render_accumulate_async(st["camera"], p, outs, stream=side)
        total = outs[2].sum()                  # queued on `side` after the render
    g.sync()
    side.synchronize()
    assert int(total) == 128 * 96 * 16
    for x, y in zip(outs, ref):
        _same(x.cpu().numpy(), y)
    stats = g.last_stats()
    assert stats["ext_rays"] > 0 and stats["ms"] > 0
    # two calls queued back to back, then one sync
    p2 = pass_params(128, 96, 16, 16, 4, 8, 4, 1.0, 7)
    g.render_accumulate_async(st["camera"], p, outs)
    g.render_accumulate_async(st["camera"], p2, outs, reset=False)
    g.sync()
    both = g.render_accumulate(st["camera"], pass_params(128, 96, 0, 32, 4, 8, 4, 1.0, 7))
    assert int(outs[2].sum()) == 128 * 96 * 32
    np.testing.assert_allclose(outs[0].cpu().numpy(), both[0], rtol=1e-5, atol=1e-6)


def test_async_errors():
    import torch
    sb, st = configs.box_scene(width=64, height=64)
    g = GpuScene(sb)
    dev = torch.device("cuda", 0)
    outs = (torch.zeros((64, 64, 3), device=dev), torch.zeros((64, 64, 3), device=dev),
            torch.zeros((64, 64), dtype=torch.int32, device=dev))
    g.set_tuning(max_iterations=2)
    g.render_accumulate_async(st["camera"], pass_params(64, 64, 0, 2, 1, 8, 4, 1.0, 9), outs)
    with pytest.raises(RtError) as e:
        g.sync()
    assert e.value.code == RT_ERR_TIMEOUT
    g.set_tuning()
    g.render_accumulate_async(st["camera"], pass_params(64, 64, 0, 2, 1, 8, 4, 1.0, 9), outs)
    g.sync()
    assert int(outs[2].sum()) == 64 * 64 * 2


def test_graph_with_the_frozen_guide_is_bit_identical():
    """The guide's encode and inference kernels inside the captured iterations:
    with the network frozen (RT_GUIDE_SAMPLE) a render is deterministic, and
    the graph form gives the host-driven loop's image bit for bit."""
    from rustracer_b200 import abi
    from rustracer_b200.renderer import guide_params
    sb, st = configs.guided_box_scene(width=64, height=48, gem=False)
    g = GpuScene(sb)
    g.guide_init(guide_params(batch=4096, steps_per_pass=2, seed=5))
    g.guide_mode(abi.RT_GUIDE_TRAIN)
    g.render_accumulate(st["camera"], pass_params(64, 48, 0, 4, 2, 12, 4, 1.0, 3))
    g.guide_mode(abi.RT_GUIDE_SAMPLE)
    p = pass_params(64, 48, 100, 8, 2, 12, 4, 1.0, 9)
    ref = g.render_pass(st["camera"], p)
    g.set_tuning(graph=1)
    _same(g.render_pass(st["camera"], p), ref)
    _same(g.render_pass(st["camera"], p), ref)      # replayed
