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
