"""Caustic photon map on the GPU against the CPU oracle: photon tracing and
storage, the gather estimates, exact k-NN neighbour sets, and rendering with
caustic injection."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200 import configs, photons
from rustracer_b200.renderer import GpuScene, RtError, pass_params
from tests.test_oracle_photons import glass_over_floor
from tests.test_gpu_render import assert_tiles_agree

pytestmark = pytest.mark.gpu


def test_gpu_photon_build_matches_oracle():
    sb = glass_over_floor()
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = photons.photon_params([photons.disk_emitter((0, 1, 0), (10, 10, 10), 20000)], 0.5, seed=1)
    ng, no = g.photon_build(p), o.photon_build(p)
    assert ng > 2000 and abs(ng - no) <= max(20, no // 100), (ng, no)
    gp, gw, gn, gi = g.photon_export()
    op, ow, on, oi = o.photon_export()
    assert (np.diff(gi) > 0).all()
    common, ga, oa = np.intersect1d(gi, oi, return_indices=True)
    assert len(common) > 0.98 * min(ng, no)
    np.testing.assert_allclose(gp[ga], op[oa], atol=1e-4)
    np.testing.assert_allclose(gw[ga], ow[oa], rtol=1e-4, atol=1e-7)


def _random_photons(n, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1, 1, size=(n, 3)).astype(np.float32)
    pos[:, 1] *= 0.05
    power = rng.uniform(0, 1, size=(n, 3)).astype(np.float32)
    nor = np.tile(np.array([0, 1, 0], np.float32), (n, 1))
    nor[::5] = (0, -1, 0)
    return pos, power, nor


@pytest.mark.parametrize("knn_k", [0, 32])
def test_gpu_gather_matches_oracle(knn_k):
    pos, power, nor = _random_photons(50000, 5)
    sb = glass_over_floor()
    g, o = GpuScene(sb), O.OracleScene(sb)
    g.photon_set(pos, power, nor, np.arange(len(pos)), radius=0.05, knn_k=knn_k)
    o.photon_set(pos, power, nor, np.arange(len(pos)), radius=0.05, knn_k=knn_k)
    rng = np.random.default_rng(6)
    q = np.zeros((3000, 6), np.float32)
    q[:, 0] = rng.uniform(-1, 1, 3000)
    q[:, 2] = rng.uniform(-1, 1, 3000)
    q[:, 4] = 1.0
    a, b = g.photon_gather(q), o.photon_gather(q)
    np.testing.assert_allclose(a, b, rtol=2e-4, atol=1e-5)
    assert (b.sum(1) > 0).mean() > 0.9


@pytest.mark.parametrize("knn_k", [0, 8])
def test_gpu_gather_on_a_coarsened_grid(knn_k):
    """Photons filling a cube with a small radius: cells of 2r would number
    over 10^8, so the grid takes larger cells (fewer than 2^22 of them); the
    estimates still match the oracle's, photon for photon."""
    rng = np.random.default_rng(11)
    n = 60000
    pos = rng.uniform(-1, 1, size=(n, 3)).astype(np.float32)
    power = rng.uniform(0, 1, size=(n, 3)).astype(np.float32)
    nor = rng.normal(size=(n, 3)).astype(np.float32)
    nor /= np.linalg.norm(nor, axis=1, keepdims=True)
    sb = glass_over_floor()
    g, o = GpuScene(sb), O.OracleScene(sb)
    g.photon_set(pos, power, nor, np.arange(n), radius=0.004, knn_k=knn_k)
    o.photon_set(pos, power, nor, np.arange(n), radius=0.004, knn_k=knn_k)
    q = np.zeros((4000, 6), np.float32)
    q[:, :3] = pos[:4000] + rng.uniform(-0.001, 0.001, size=(4000, 3))
    q[:, 3:] = nor[:4000]
    a, b = g.photon_gather(q), o.photon_gather(q)
    np.testing.assert_allclose(a, b, rtol=2e-4, atol=1e-5)
    assert (b.sum(1) > 0).mean() > 0.9
    i1, d1 = g.knn(q[:, :3], 8, 0.004)
    i2, d2 = o.knn(q[:, :3], 8, 0.004)
    assert np.array_equal(i1, i2)


def test_gpu_knn_sets_are_exact():
    pos, power, nor = _random_photons(40000, 7)
    pos = (np.round(pos * 64) / 64).astype(np.float32)          # exact distance ties
    sb = glass_over_floor()
    g, o = GpuScene(sb), O.OracleScene(sb)
    g.photon_set(pos, power, nor, np.arange(len(pos)), radius=0.1)
    o.photon_set(pos, power, nor, np.arange(len(pos)), radius=0.1)
    rng = np.random.default_rng(8)
    q = rng.uniform(-1, 1, size=(2000, 3)).astype(np.float32)
    q[:, 1] *= 0.05
    # radii up to the map's (0.1) use its cell grid, 0.2 the box heap
    for k, rmax in [(64, 0.01), (16, 0.05), (64, 0.05), (64, 0.1), (16, 0.2)]:
        gi, gd = g.knn(q, k, rmax)
        oi, od = o.knn(q, k, rmax)
        assert np.array_equal(gi, oi), (k, rmax)
        fin = np.isfinite(od)
        assert np.array_equal(gd[fin].view(np.uint32), od[fin].view(np.uint32))


def test_gpu_render_with_caustics_matches_oracle():
    sb, st = configs.box_scene(width=64, height=64)
    p = photons.caustic_params(sb, 200000, 0.05, seed=2)
    g, o = GpuScene(sb), O.OracleScene(sb)
    ng, no = g.photon_build(p), o.photon_build(p)
    assert ng > 1000 and abs(ng - no) <= max(20, no // 50)
    pp = pass_params(64, 64, 0, 64, 8, 8, 4, 1.0, 3)
    gi = g.render_pass(st["camera"], pp)
    pp.seed = 4
    oi = o.render_pass(st["camera"], pp)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)
    g.photon_clear()
    assert g.photon_export()[0].shape[0] == 0


def test_gpu_photon_errors():
    g = GpuScene(glass_over_floor())
    p = photons.photon_params([photons.disk_emitter((0, 1, 0), (1, 1, 1), 100)], 0.0)
    with pytest.raises(RtError):
        g.photon_build(p)
