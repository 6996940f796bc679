"""Cylinders, cones, disks and infinite planes on the GPU against the CPU
oracle: identical hit ids, t and surface part (placed by scale, rotation and
translation), and render tiles within 3 SE."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.renderer import GpuScene, pass_params
from rustracer_b200.scene import Material, SceneBuilder, Transform, make_camera
from tests.helpers import camera_rays, random_rays
from tests.test_gpu_render import assert_tiles_agree
from tests.test_gpu_trace import assert_same_hits

pytestmark = pytest.mark.gpu


def shape_field():
    sb = SceneBuilder()
    floor = sb.add_material(Material.pbr((0.5, 0.48, 0.46), roughness=0.25))
    red = sb.add_material(Material.lambertian((0.7, 0.2, 0.15)))
    glass = sb.add_material(Material.dielectric(1.5))
    gold = sb.add_material(Material.spectral_metal("gold", 0.2))
    water = sb.add_material(Material.lambertian((0.2, 0.35, 0.5)))
    sb.add_shape("disk", floor, (0, 0, 0), radius=6.0, normal=(0, 1, 0))
    sb.add_shape("infinite_plane", water, (0, -0.2, 0), normal=(0, 1, 0), wave_amplitude=0.05, wave_scale=4.0)
    sb.add_shape("cylinder", red, (-1.2, 0, 0), radius=0.4, height=1.0)
    sb.add_shape("cone", gold, (0.0, 0, -0.5), radius=0.5, height=1.2)
    sb.add_shape("cylinder", glass, (0, 0, 0), radius=0.3, height=0.8,
                 xf=Transform(scale=1.2, rotate=(70.0, 20.0, 0.0), translate=(1.2, 0.5, 0.3)))
    sb.add_shape("disk", red, (0, 0, 0), radius=0.35, normal=(0.3, 1.0, -0.2),
                 xf=Transform(rotate=(0.0, 0.0, 60.0), translate=(-0.2, 0.9, 0.9)))
    sb.add_sphere((0.6, 0.3, 0.8), 0.3, glass)
    light = sb.add_material(Material.diffuse_light((10.0, 10.0, 10.0)))
    sb.add_light_quad((-0.75, 3.0, -0.75), (1.5, 0, 0), (0, 0, 1.5), light)
    sb.set_physical(40.0, 30.0, 3.0)
    return sb


def test_gpu_shape_trace_matches_oracle():
    sb = shape_field()
    g, o = GpuScene(sb), O.OracleScene(sb)
    rs = np.concatenate([random_rays(60000, 13, center=(0, 0.5, 0), radius=3.0, spread=0.8),
                         camera_rays(make_camera((0.0, 1.8, 4.0), (0.0, 0.4, 0.0), vfov=40.0, aspect=1.0), 128, 128)])
    gh, oh = g.trace_closest(rs), o.trace_closest(rs)
    assert (oh["prim"] >= 2).sum() > 5000
    assert_same_hits(gh, oh)
    assert np.array_equal(g.trace_any(rs), o.trace_any(rs))


@pytest.mark.parametrize("hero", [1, 4])
def test_gpu_shape_render_matches_oracle(hero):
    sb = shape_field()
    sb.spectral_range = 1 if hero > 1 else 0
    cam = make_camera((0.0, 1.8, 4.0), (0.0, 0.4, 0.0), vfov=40.0, aspect=1.0)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = pass_params(64, 64, 0, 64, 8, 10, hero, 1.0, 61)
    gi = g.render_pass(cam, p)
    p.seed = 62
    oi = o.render_pass(cam, p)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)
