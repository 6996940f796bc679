"""Batched rendering on concurrent scene handles: every frame equals the same
frame rendered alone (the render is deterministic per seed and sample)."""
import numpy as np
import pytest

from rustracer_b200 import batch, configs

pytestmark = pytest.mark.gpu


def test_concurrent_batch_matches_sequential():
    jobs = batch.make_jobs(seed=5, n=8, scenes=("box",), min_width=32, max_width=96, min_spp=2, max_spp=8)
    sb = {"box": configs.box_scene()[0]}
    par = batch.run_batch(jobs, workers=3, builders=sb, keep_outputs=True)
    seq = batch.run_batch(jobs, workers=1, builders=sb, keep_outputs=True)
    for j in jobs:
        a, b = par["outputs"][j["id"]], seq["outputs"][j["id"]]
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    assert par["path_samples"] == sum(j["width"] * j["height"] * j["spp"] for j in jobs)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("graph", [False, True])
def test_packed_batch_frames_are_bit_identical_to_single_renders(graph):
    """Requests of different size, spp, camera and seed packed into one
    wavefront pool (rt_render_batch, in passes of 3 samples per pixel so most
    requests span several passes) give every request exactly the sum, M2 and
    count of rendering it alone with rt_render_accumulate, whether the passes
    run the host-driven loop or replay the captured wavefront graph."""
    jobs = batch.make_jobs(seed=7, n=10, scenes=("box", "icosphere"), min_width=24, max_width=80, min_spp=1, max_spp=9)
    builders = {"box": configs.box_scene()[0], "icosphere": configs.icosphere_scene(levels=4, env_w=64, env_h=32)[0]}
    packed = batch.run_packed(jobs, builders=builders, keep_outputs=True, window=3, graph=graph)
    seq = batch.run_batch(jobs, workers=1, builders=builders, keep_outputs=True)
    for j in jobs:
        a, b = packed["outputs"][j["id"]], seq["outputs"][j["id"]]
        for x, y in zip(a, b):
            assert x.shape == y.shape
            assert np.array_equal(_bits(x), _bits(y)), j
    assert all(0 < packed["latencies"][j["id"]] <= packed["wall_s"] + 1e-3 for j in jobs)


def test_packed_batch_single_pass_and_device_outputs():
    """window 0 (as many samples per pass as fit) and CUDA-tensor outputs."""
    import torch
    from rustracer_b200.renderer import GpuScene, pass_params
    sb, st = configs.box_scene(width=48, height=40)
    g = GpuScene(sb)
    reqs = [dict(cam=st["camera"], width=48, height=40, spp=5, seed=3),
            dict(cam=st["camera"], width=17, height=9, spp=2, seed=4, sample_idx=6)]
    tot = 48 * 40 + 17 * 9
    outs = (torch.zeros(tot * 3, device="cuda"), torch.zeros(tot * 3, device="cuda"),
            torch.zeros(tot, dtype=torch.int32, device="cuda"))
    res, done = g.render_batch(reqs, pass_params(8, 8, 0, 1, 1, 8, 4, 1.0, 0), outputs=outs)
    torch.cuda.synchronize()
    assert (done > 0).all()
    for r, q in zip(res, reqs):
        s1, m1, c1 = g.render_accumulate(q["cam"], pass_params(q["width"], q["height"], q.get("sample_idx", 0),
                                                               q["spp"], int(np.sqrt(q["spp"])), 8, 4, 1.0, q["seed"]))
        assert np.array_equal(_bits(r[0].cpu().numpy()), _bits(s1))
        assert np.array_equal(_bits(r[1].cpu().numpy()), _bits(m1))
        assert np.array_equal(r[2].cpu().numpy().astype(np.uint32), c1)
