"""Ray-level parity of the CUDA traversal against the CPU oracle: identical
canonical primitive ids and bit-identical t / barycentrics, plus the
reference's primitive known-answer tests run through the GPU entry points."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200 import configs
from rustracer_b200.renderer import GpuScene, RtError
from rustracer_b200.scene import Material, SceneBuilder
from tests.helpers import camera_rays, random_rays, ray, rays, spheres_scene, unit_quad_scene, xy_triangle_scene

pytestmark = pytest.mark.gpu


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def assert_same_hits(g, o):
    assert np.array_equal(g["prim"], o["prim"]), np.flatnonzero(g["prim"] != o["prim"])[:10]
    hit = o["prim"] >= 0
    for f in ("t", "b1", "b2"):
        assert np.array_equal(bits(g[f][hit]), bits(o[f][hit])), f


# ── known answers (quad.rs / triangle.rs / sphere.rs / bvh.rs tests) ─────────
def test_gpu_quad_known_answers():
    s = GpuScene(unit_quad_scene())
    h = s.trace_closest(rays(
        ray((0.5, 0.5, 3.0), (0, 0, -1)), ray((0.25, 0.75, 1.0), (0, 0, -1)),
        ray((0, 0, 1), (0, 0, -1)), ray((1, 0, 1), (0, 0, -1)), ray((0, 1, 1), (0, 0, -1)), ray((1, 1, 1), (0, 0, -1)),
        ray((1.01, 0.5, 1.0), (0, 0, -1)), ray((0.5, -0.01, 1.0), (0, 0, -1)), ray((0.5, 0.5, 0.0), (1, 0, 0))))
    assert abs(h["t"][0] - 3.0) < 1e-5
    assert abs(h["b1"][1] - 0.25) < 1e-5 and abs(h["b2"][1] - 0.75) < 1e-5
    assert (h["prim"][2:6] == 0).all() and (h["prim"][6:] == -1).all()


def test_gpu_triangle_known_answers():
    s = GpuScene(xy_triangle_scene())
    h = s.trace_closest(rays(
        ray((2 / 3, 2 / 3, -5.0), (0, 0, 1)), ray((0.0, 0.0, -3.0), (0, 0, 1)), ray((3.0, 0.0, -1.0), (0, 0, 1)),
        ray((0.0, -1.0, -1.0), (0, 0, 1)), ray((1.5, 1.5, -1.0), (0, 0, 1)), ray((0.5, 0.5, 0.0), (1, 0, 0)),
        ray((2 / 3, 2 / 3, -1.0), (0, 0, 1))))
    assert abs(h["t"][0] - 5.0) < 1e-5 and abs(h["t"][1] - 3.0) < 1e-5
    assert (h["prim"][2:6] == -1).all()
    assert abs(h["b1"][6] - 1 / 3) < 1e-5 and abs(h["b2"][6] - 1 / 3) < 1e-5


def test_gpu_sphere_and_bvh_known_answers():
    s = GpuScene(spheres_scene([(0, 0, 0)]))
    h = s.trace_closest(rays(ray((0, 0, -5), (0, 0, 0)), ray((0, 0, -5), (0, 0, 1)), ray((2, 0, -5), (0, 0, 1))))
    assert list(h["prim"]) == [-1, 0, -1]
    assert list(s.trace_any(rays(ray((0, 0, -5), (0, 0, 1)), ray((2, 0, -5), (0, 0, 1))))) == [1, 0]
    two = GpuScene(spheres_scene([(0, 0, -3), (0, 0, 3)]))
    assert two.trace_closest(rays(ray((0, 0, -10), (0, 0, 1))))["t"][0] < 8.0
    pos = [(x * 10.0, y * 10.0, 0.0) for x in (-1, 0, 1) for y in (-1, 0, 1)]
    grid = GpuScene(spheres_scene(pos))
    assert (grid.trace_closest(rays(*[ray((p[0], p[1], -20.0), (0, 0, 1)) for p in pos]))["prim"] >= 0).all()


def test_gpu_closed_interval_and_tmax():
    # hittable.rs:97-101: a hit at exactly t == t_max is accepted
    s = GpuScene(unit_quad_scene())
    h = s.trace_closest(rays(ray((0.5, 0.5, 3.0), (0, 0, -1), 0.001, 3.0), ray((0.5, 0.5, 3.0), (0, 0, -1), 0.001, 2.999)))
    assert list(h["prim"]) == [0, -1]


def test_gpu_rejects_degenerate_and_empty_input():
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((1, 1, 1)))
    sb.add_quad((0, 0, 0), (1, 0, 0), (2, 0, 0), m)
    with pytest.raises(RtError) as e:
        GpuScene(sb)
    assert e.value.code == 1 and "degenerate" in str(e.value)
    bad = SceneBuilder()
    bad.add_sphere((0, 0, 0), 1.0, 3)   # material index out of range
    with pytest.raises(RtError):
        GpuScene(bad)
    empty = GpuScene(SceneBuilder())
    h = empty.trace_closest(rays(ray((0, 0, 0), (0, 0, 1))))
    assert h["prim"][0] == -1


# ── BVH: a valid 8-wide tree over the reference's SAH partitions ─────────────
def sah_cost(nodes):
    """Σ inner-node area + Σ leaf area, normalised by the root area (8-wide
    nodes in the reference layout: min[3][8], max[3][8], children[8])."""
    mn = nodes[:, 0:24].reshape(-1, 3, 8)
    mx = nodes[:, 24:48].reshape(-1, 3, 8)
    ch = nodes[:, 48:56].view(np.int32)
    valid = ch != np.iinfo(np.int32).min
    area = lambda lo, hi: 2 * ((hi[:, 0] - lo[:, 0]) * (hi[:, 1] - lo[:, 1]) + (hi[:, 1] - lo[:, 1]) * (hi[:, 2] - lo[:, 2])
                               + (hi[:, 2] - lo[:, 2]) * (hi[:, 0] - lo[:, 0]))
    big = np.float64(1e30)
    nlo = np.where(valid[:, None, :], mn, big).min(axis=2)
    nhi = np.where(valid[:, None, :], mx, -big).max(axis=2)
    node_area = area(nlo.astype(np.float64), nhi.astype(np.float64))
    leaf = valid & (ch < 0)
    leaf_area = area(mn.transpose(0, 2, 1)[leaf].astype(np.float64), mx.transpose(0, 2, 1)[leaf].astype(np.float64))
    return (node_area.sum() + leaf_area.sum()) / node_area[0]


def check_tree(nodes, leaves, n_prims):
    ch = nodes[:, 48:56].view(np.int32)
    valid = ch != np.iinfo(np.int32).min
    assert sorted(leaves.tolist()) == list(range(n_prims))            # every primitive exactly once
    slots = -ch[valid & (ch < 0)] - 1
    assert sorted(slots.tolist()) == list(range(len(leaves)))
    inner = ch[valid & (ch >= 0)]
    assert sorted(inner.tolist()) == list(range(1, len(nodes)))       # every node but the root has one parent
    mn = nodes[:, 0:24].reshape(-1, 3, 8)
    mx = nodes[:, 24:48].reshape(-1, 3, 8)
    for i, c in zip(*np.nonzero(valid & (ch >= 0))):                  # child box == union of its node's boxes
        k = ch[i, c]
        kv = valid[k]
        assert np.array_equal(mn[i, :, c], mn[k][:, kv].min(axis=1))
        assert np.array_equal(mx[i, :, c], mx[k][:, kv].max(axis=1))


@pytest.mark.parametrize("name", ["box", "ico5"])
def test_gpu_bvh_is_valid_and_no_worse_than_reference(name):
    if name == "box":
        sb, _ = configs.box_scene()
    else:
        sb, _ = configs.icosphere_scene(levels=5, env_w=64, env_h=32)
    g, o = GpuScene(sb), O.OracleScene(sb)
    gn, gl = g.bvh()
    on, ol = o.bvh()
    n = sb.n_tris + len(sb.quads) + len(sb.spheres)
    check_tree(gn, gl, n)
    check_tree(on, ol, n)
    assert sah_cost(gn) <= sah_cost(on) * 1.0001
    st = g.bvh_stats()
    assert st["nodes"] == len(gn) and st["leaves"] == n
    if name == "ico5":
        assert len(gn) < len(on)              # fuller 8-wide nodes than the fixed 3-level split


# ── hit parity on random and camera rays ─────────────────────────────────────
def test_gpu_hits_match_oracle_icosphere():
    sb, st = configs.icosphere_scene(levels=6, env_w=64, env_h=32)
    g, o = GpuScene(sb), O.OracleScene(sb)
    r = np.concatenate([random_rays(60000, 11, spread=0.6), camera_rays(st["camera"], 192, 108, seed=2)])
    gh, oh = g.trace_closest(r), o.trace_closest(r)
    assert_same_hits(gh, oh)
    assert (oh["prim"] >= 0).mean() > 0.3
    sub = r[:5000]
    assert_same_hits(gh[:5000], o.trace_closest(sub, brute=True))
    assert np.array_equal(g.trace_any(r), o.trace_any(r))


def test_gpu_hits_match_oracle_box_and_edges():
    sb, st = configs.box_scene()
    g, o = GpuScene(sb), O.OracleScene(sb)
    r = np.concatenate([camera_rays(st["camera"], 128, 128, seed=5), random_rays(20000, 5, center=(0.5, 0.5, 0.5),
                                                                                   radius=0.4, spread=0.5)])
    # axis-aligned rays through edges and corners of the room, and degenerate rays
    edge = [ray((x, y, -1.0), (0, 0, 1)) for x in (0.0, 0.5, 1.0) for y in (0.0, 0.5, 1.0)]
    edge += [ray((0.5, 0.5, 0.5), (0, 0, 0)), ray((np.nan, 0.5, 0.5), (0, 0, 1)), ray((0.5, 0.5, 0.5), (1, 0, 0), 0.001, 0.2)]
    r = np.concatenate([r, rays(*edge)])
    assert_same_hits(g.trace_closest(r), o.trace_closest(r))
    assert_same_hits(g.trace_closest(r[-12:]), o.trace_closest(r[-12:], brute=True))
    assert np.array_equal(g.trace_any(r), o.trace_any(r))


def test_gpu_hits_full_icosphere_config():
    """1,310,720-triangle icosphere of the benchmark workload: 100k rays."""
    sb, st = configs.icosphere_scene(env_w=64, env_h=32)
    g, o = GpuScene(sb), O.OracleScene(sb)
    r = np.concatenate([random_rays(50000, 21, spread=0.7), camera_rays(st["camera"], 320, 160, seed=9)])
    assert_same_hits(g.trace_closest(r), o.trace_closest(r))
    assert np.array_equal(g.trace_any(r), o.trace_any(r))
