"""Limits of the device loops and the traversal stack, and the node layouts.

The traversal stack keeps its newest entries in a per-thread ring and
spills deeper ones to global memory, so no scene's tree overflows it (the
reference keeps 128 entries inline and spills to a heap Vec, bvh.rs:229-239).
rt_set_tuning can shrink the ring, which sends every traversal through the
spill path: the hits must not change.  It can also lower the stack capacity
and the wavefront's iteration bound, which makes the library return
RT_ERR_CAPACITY / RT_ERR_TIMEOUT from a render or trace call instead of
faulting, and leaves the scene usable."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200 import configs
from rustracer_b200.renderer import GpuScene, RtError, pass_params
from tests.helpers import camera_rays, random_rays

pytestmark = pytest.mark.gpu

RT_ERR_CAPACITY, RT_ERR_TIMEOUT = 2, 3


def _hits_equal(a, b):
    assert np.array_equal(a["prim"], b["prim"]), np.flatnonzero(a["prim"] != b["prim"])[:10]
    hit = a["prim"] >= 0
    for f in ("t", "b1", "b2"):
        assert np.array_equal(a[f][hit].view(np.uint32), b[f][hit].view(np.uint32)), f


def test_spilled_stack_gives_the_same_hits_on_the_icosphere():
    """1.31M-triangle icosphere: with a ring of 1 or 2 slots nearly every push
    and pop goes through the global spill columns; hits, t and barycentrics
    stay bit-identical to the 16-slot ring and to the oracle."""
    sb, st = configs.icosphere_scene(env_w=64, env_h=32)
    g, o = GpuScene(sb), O.OracleScene(sb)
    r = np.concatenate([random_rays(30000, 31, spread=0.7), camera_rays(st["camera"], 200, 100, seed=4)])
    assert g.get_tuning()["stack_ring"] == 16
    base = g.trace_closest(r)
    base_any = g.trace_any(r)
    _hits_equal(base[:8000], o.trace_closest(r[:8000]))
    for ring in (1, 2, 8):
        g.set_tuning(stack_ring=ring)
        _hits_equal(g.trace_closest(r), base)
        assert np.array_equal(g.trace_any(r), base_any)
    g.set_tuning()
    assert g.get_tuning()["stack_ring"] == 16


def test_spilled_stack_renders_the_same_image():
    """A render pass (extend and shadow kernels of the wavefront) with a
    one-slot ring is bit-identical to the default."""
    sb, st = configs.box_scene(width=96, height=96)
    g = GpuScene(sb)
    p = pass_params(96, 96, 0, 4, 2, 8, 4, 1.0, 17)
    a = g.render_pass(st["camera"], p)
    g.set_tuning(stack_ring=1)
    b = g.render_pass(st["camera"], p)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_stack_capacity_error_is_returned_and_the_scene_stays_usable():
    sb, st = configs.icosphere_scene(env_w=64, env_h=32)
    g = GpuScene(sb)
    cap = g.get_tuning()["stack_limit"]
    depth = g.bvh_stats()["max_depth"]
    assert cap == 7 * (depth + 1) + 8
    r = random_rays(4096, 5, spread=0.7)
    ref = g.trace_closest(r)
    g.set_tuning(stack_limit=1)
    with pytest.raises(RtError) as e:
        g.trace_closest(r)
    assert e.value.code == RT_ERR_CAPACITY
    with pytest.raises(RtError) as e:
        g.render_pass(st["camera"], pass_params(64, 36, 0, 1, 1, 12, 4, 1.0, 2))
    assert e.value.code == RT_ERR_CAPACITY
    with pytest.raises(RtError) as e:
        g.set_tuning(stack_limit=cap + 1)
    assert e.value.code == 1
    g.set_tuning()
    _hits_equal(g.trace_closest(r), ref)


def test_iteration_bound_returns_timeout_and_the_scene_stays_usable():
    sb, st = configs.box_scene(width=64, height=64)
    g = GpuScene(sb)
    p = pass_params(64, 64, 0, 2, 1, 8, 4, 1.0, 9)
    ref = g.render_pass(st["camera"], p)
    g.set_tuning(max_iterations=2)
    with pytest.raises(RtError) as e:
        g.render_pass(st["camera"], p)
    assert e.value.code == RT_ERR_TIMEOUT and "iteration bound" in str(e.value)
    with pytest.raises(RtError) as e:
        g.render_accumulate(st["camera"], p)
    assert e.value.code == RT_ERR_TIMEOUT
    g.set_tuning()
    assert np.array_equal(g.render_pass(st["camera"], p).view(np.uint32), ref.view(np.uint32))


def test_node_layouts_give_identical_hits_and_images():
    """The quantised 128-byte nodes (8-bit child boxes rounded outward, a
    conservative slab test), the 4-wide 112-byte nodes over the same binary
    tree (bvh.rs:10-14's other width) and the reference's 224-byte float nodes
    give the same hits bit for bit, hence the same image; the oracle agrees."""
    sb, st = configs.icosphere_scene(env_w=64, env_h=32)
    g, o = GpuScene(sb), O.OracleScene(sb)
    assert g.get_tuning()["node_format"] == 0          # the full layout is the default
    r = np.concatenate([random_rays(30000, 41, spread=0.7), camera_rays(st["camera"], 200, 100, seed=6)])
    q = g.trace_closest(r)
    qa = g.trace_any(r)
    _hits_equal(q[:8000], o.trace_closest(r[:8000]))
    p = pass_params(64, 36, 0, 2, 1, 12, 4, 1.0, 3)
    cam = configs.make_camera((0.0, 0.45, 3.6), (0.0, -0.15, 0.0), vfov=40.0, aspect=64 / 36)
    full = g.render_pass(cam, p)
    for fmt in (1, 2):                                 # quantised, 4-wide
        g.set_tuning(node_format=fmt)
        assert g.get_tuning()["node_format"] == fmt
        _hits_equal(g.trace_closest(r), q)
        assert np.array_equal(g.trace_any(r), qa)
        assert np.array_equal(g.render_pass(cam, p).view(np.uint32), full.view(np.uint32))
    # the 4-wide tree through a two-slot stack ring (every traversal spills)
    g.set_tuning(node_format=2, stack_ring=2)
    _hits_equal(g.trace_closest(r), q)
    g.set_tuning()


def test_wide4_nodes_need_a_device_built_tree():
    from rustracer_b200 import abi
    sb, _ = configs.box_scene(width=32, height=32)
    sb.bvh_builder = abi.RT_BVH_HOST
    g = GpuScene(sb)
    with pytest.raises(RtError):
        g.set_tuning(node_format=2)
    assert g.get_tuning()["node_format"] == 0


@pytest.mark.parametrize("name", ["media_box", "gem_room"])
def test_node_layouts_render_identically_with_media_and_solids(name):
    """The traversal instantiations with analytic solids (the gem room's
    [[gems]] stones and shapes) and the media shadow mode read every layout
    the same way: renders are bit-identical."""
    if name == "media_box":
        sb, st = configs.media_box_scene(width=48, height=48)
    else:
        sb, st = configs.gem_room_scene(48, 32)
    g = GpuScene(sb)
    p = pass_params(48, 48 if name == "media_box" else 32, 0, 4, 2, 12, 4, 1.0, 17)
    ref = g.render_pass(st["camera"], p)
    for fmt in (1, 2):
        try:
            g.set_tuning(node_format=fmt)
        except RtError:
            continue                                   # a layout this scene lacks
        assert np.array_equal(g.render_pass(st["camera"], p).view(np.uint32), ref.view(np.uint32)), fmt
    g.set_tuning()
