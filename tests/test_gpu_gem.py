"""The gem workload (round brilliant in dispersive diamond, two blackbody
lights, dim sky, k-NN caustic photon map) on the GPU against the CPU oracle,
at a reduced size."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200 import configs, photons
from rustracer_b200.renderer import GpuScene, pass_params
from tests.test_gpu_render import assert_tiles_agree

pytestmark = pytest.mark.gpu


def test_gpu_gem_scene_matches_oracle():
    sb, st = configs.gem_scene(width=96, height=54)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = photons.caustic_params(sb, 1_000_000, st["radius_max"], knn_k=st["knn_k"], seed=1, env_dir=st["env_dir"],
                               env_color=st["env_color"])
    ng, no = g.photon_build(p), o.photon_build(p)
    assert ng > 1000 and abs(ng - no) <= max(30, no // 20), (ng, no)
    pp = pass_params(96, 54, 0, 64, 8, st["max_depth"], st["hero"], 1.0, 41)
    gi = g.render_pass(st["camera"], pp)
    pp.seed = 42
    oi = o.render_pass(st["camera"], pp)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)
