"""The gem workload (57-facet round brilliant in dispersive diamond, two
blackbody lights, dim sky, k-NN caustic photon map emitted from the lights
toward the stone) on the GPU against the CPU oracle: the dense photon map
(counts, positions) at the workload's 2M photons, and render tiles at a
reduced frame size."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200 import configs, photons
from rustracer_b200.renderer import GpuScene, pass_params
from tests.test_gpu_render import assert_tiles_agree

pytestmark = pytest.mark.gpu


def test_gpu_gem_dense_photon_map_matches_oracle():
    """2M photons from the two lights toward the stone: 10^5-10^6 stored,
    within 1 % of the oracle's count, and the photons both sides store for
    the same emission index lie at the same place."""
    sb, st = configs.gem_scene(width=96, height=54)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = st["photon_params"](seed=1)
    assert sum(p.emitters[i].n_photons for i in range(p.n_emitters)) == 2_000_000
    ng, no = g.photon_build(p), o.photon_build(p)
    assert 100_000 <= ng <= 1_000_000, ng
    assert abs(ng - no) <= no // 100, (ng, no)
    gp, gw, gn, gi = g.photon_export()
    op, ow, on, oi = o.photon_export()
    common, ga, oa = np.intersect1d(gi, oi, return_indices=True)
    assert len(common) >= 0.98 * no
    close = np.linalg.norm(gp[ga] - op[oa], axis=1) < 1e-4
    assert close.mean() > 0.99, close.mean()
    assert np.allclose(gw.sum(0), ow.sum(0), rtol=0.02)


def test_gpu_photon_shards_rebuild_the_full_map():
    """Two shards of the emission order, traced separately and joined with
    rt_photon_set, give the unsharded build's photons bit for bit (the
    exchange a multi-GPU render makes)."""
    sb, st = configs.gem_scene(width=96, height=54)
    g = GpuScene(sb)
    p = st["photon_params"](seed=4, n=400_000)
    g.photon_build(p)
    ref = g.photon_export()
    parts = []
    for r in range(2):
        g.photon_build(photons.shard_params(p, 2, r))
        parts.append(g.photon_export())
    for k in range(4):
        joined = np.concatenate([q[k] for q in parts])
        assert np.array_equal(joined.view(np.uint32) if joined.dtype == np.float32 else joined,
                              ref[k].view(np.uint32) if ref[k].dtype == np.float32 else ref[k])
    pos, pw, nor, idx = (np.concatenate([q[k] for q in parts]) for k in range(4))
    g.photon_set(pos, pw, nor, idx, radius=st["radius_max"], knn_k=st["knn_k"])
    q = pos[:: max(1, len(pos) // 2000)]
    i1, d1 = g.knn(q, 16, st["radius_max"])
    g.photon_build(p)
    i2, d2 = g.knn(q, 16, st["radius_max"])
    assert np.array_equal(i1, i2) and np.array_equal(d1.view(np.uint32), d2.view(np.uint32))


def test_gpu_gem_scene_matches_oracle():
    sb, st = configs.gem_scene(width=96, height=54)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = st["photon_params"](seed=1, n=1_000_000)
    ng, no = g.photon_build(p), o.photon_build(p)
    assert ng > 50_000 and abs(ng - no) <= max(30, no // 100), (ng, no)
    pp = pass_params(96, 54, 0, 64, 8, st["max_depth"], st["hero"], 1.0, 41)
    gi = g.render_pass(st["camera"], pp)
    pp.seed = 42
    oi = o.render_pass(st["camera"], pp)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)


def test_gem_config_band_at_its_stated_size():
    """The gem workload at its stated frame, 1280×720, depth 32, hero 4, with
    its 2M-photon caustic map (each side builds its own from the same seed):
    a 32-row band through the stone and its caustic, tiles within 3 SE."""
    sb, st = configs.gem_scene()
    assert (st["width"], st["height"], st["max_depth"], st["hero"]) == (1280, 720, 32, 4)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = st["photon_params"](seed=1)
    ng, no = g.photon_build(p), o.photon_build(p)
    assert abs(ng - no) <= no // 100
    pp = pass_params(1280, 720, 0, 32, 4, 32, 4, 1.0, 51)
    gi = g.render_pass(st["camera"], pp)
    pp.seed = 52
    oi = o.render_pass(st["camera"], pp, rows=(384, 416))
    assert gi.shape == (32, 720, 1280, 3) and np.isfinite(gi).all()
    z = assert_tiles_agree(gi[:, 384:416], oi[:, 384:416])
    assert z.size == 2 * 80
