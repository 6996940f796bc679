"""The device BVH builder (rt_build.cu: the binary SAH tree and its collapse
to 8-wide nodes on the device) against the host builder: the same binary SAH
partition (bvh.rs:290-323) and the same greedy collapse, so the exported node
boxes, children, leaf order and tree statistics are equal, and both node
layouts of both builds trace the same hits, for large triangle meshes, random
soups, degenerate clusters and mixed scenes."""
import numpy as np
import pytest

from rustracer_b200 import abi, configs
from rustracer_b200.renderer import GpuScene
from rustracer_b200.scene import Material, SceneBuilder
from tests.helpers import spheres_scene

pytestmark = pytest.mark.gpu


def _tri_soup(n, seed, spread=10.0, size=0.3):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 3))
    V = (c[:, None, :] + rng.normal(0, size, (n, 3, 3))).reshape(-1, 3)
    sb = SceneBuilder()
    sb.add_mesh(V, np.arange(3 * n).reshape(-1, 3), sb.add_material(Material.lambertian((0.5, 0.5, 0.5))))
    return sb


def _clusters(seed):
    """Many coincident triangles (degenerate centroid extents) plus a few far ones."""
    rng = np.random.default_rng(seed)
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], float)
    V = [tri] * 3000 + [tri + rng.uniform(-50, 50, 3) for _ in range(500)]
    sb = SceneBuilder()
    sb.add_mesh(np.concatenate(V), np.arange(3 * len(V)).reshape(-1, 3),
                sb.add_material(Material.lambertian((0.5, 0.5, 0.5))))
    return sb


def _same_bvh(sb):
    sb.bvh_builder = abi.RT_BVH_HOST
    host = GpuScene(sb)
    hn, hl = host.bvh()
    sb.bvh_builder = abi.RT_BVH_DEVICE
    dev = GpuScene(sb)
    dn, dl = dev.bvh()
    assert hn.shape == dn.shape and np.array_equal(hl, dl)
    assert (hn[:, :48] == dn[:, :48]).all()       # child boxes: equal values (a zero may differ in sign)
    assert np.array_equal(hn[:, 48:].view(np.uint32), dn[:, 48:].view(np.uint32))   # child references
    hs, ds = host.bvh_stats(), dev.bvh_stats()
    assert (hs["nodes"], hs["leaves"], hs["max_depth"]) == (ds["nodes"], ds["leaves"], ds["max_depth"])
    assert abs(hs["sah_cost"] - ds["sah_cost"]) <= 1e-9 * hs["sah_cost"]
    # every node layout of both builds traces the same hits (the 4-wide nodes
    # exist for the device build only)
    lo, hi = hn[:, :24].min(), hn[:, 24:48].max()
    rng = np.random.default_rng(5)
    o = rng.uniform(lo, hi, (4096, 3))
    d = rng.normal(size=(4096, 3))
    r = np.concatenate([o, d, np.full((4096, 1), 0.001), np.full((4096, 1), np.inf)], 1).astype(np.float32)
    ref = host.trace_closest(r)
    for g in (host, dev):
        for fmt in ((0, 1) if g is host else (0, 1, 2)):
            g.set_tuning(node_format=fmt)
            h = g.trace_closest(r)
            assert np.array_equal(h["prim"], ref["prim"]) and np.array_equal(h["t"].view(np.uint32), ref["t"].view(np.uint32))
        g.set_tuning()
    return host, dev


@pytest.mark.parametrize("make", [lambda: _tri_soup(200_000, 1), lambda: _tri_soup(5_000, 2, spread=1.0),
                                  lambda: _clusters(3), lambda: spheres_scene([(x, 0, 0) for x in range(7)]),
                                  lambda: configs.box_scene()[0], lambda: configs.gem_room_scene(96, 64)[0]])
def test_device_and_host_builders_agree(make):
    _same_bvh(make())


def test_icosphere_workload_build():
    sb, _ = configs.icosphere_scene(width=64, height=36)
    host, dev = _same_bvh(sb)
    assert dev.build_time_ms() > 0 and host.build_time_ms() > 0
