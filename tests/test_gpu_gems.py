"""Analytic convex gems on the GPU against the CPU oracle: identical hit ids,
t and crossing planes for placed round/oval brilliants (diamond.rs:202-253,
transform.rs), occlusion, renders through polished spectral gems, and caustic
photons refracted by a [[gems]] stone under a physical sky."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200 import photons
from rustracer_b200.renderer import GpuScene, pass_params
from rustracer_b200.scene import Material, SceneBuilder, make_camera, scene_from_toml_dict
from tests.helpers import camera_rays, random_rays, ray, rays
from tests.test_gpu_render import assert_tiles_agree
from tests.test_gpu_trace import assert_same_hits

pytestmark = pytest.mark.gpu


def gem_field():
    """Five placed brilliants (round, oval, faceted girdle, knife edge, scaled
    and tilted) on a floor, with a sphere and a light."""
    sb = SceneBuilder()
    floor = sb.add_material(Material.lambertian((0.6, 0.6, 0.6)))
    dia = sb.add_material(Material.spectral_dielectric_cauchy(2.351, 0.0230))
    ruby = sb.add_material(Material.spectral_dielectric_cauchy(1.741, 0.0094, (2.5, 55.0, 45.0)))
    sb.add_quad((-4, 0, -4), (8, 0, 0), (0, 0, 8), floor)
    sb.add_sphere((1.6, 0.35, -1.2), 0.35, floor)
    sb.add_diamond((0.0, 0.55, 0.0), 0.5, dia, polish=0.02, rotate=(12.0, 30.0, 0.0))
    sb.add_diamond((-1.3, 0.45, 0.4), 0.35, ruby, oval_ratio=1.4, girdle_facets=64, rotate=(0.0, -20.0, 8.0))
    sb.add_diamond((1.1, 0.4, 0.9), 0.35, dia, girdle_finish="faceted", polish=0.05)
    sb.add_diamond((-0.4, 0.3, 1.3), 0.25, dia, girdle_pct=0.0, rotate=(90.0, 0.0, 0.0))
    sb.add_diamond((0.5, 0.2, -1.1), 0.2, ruby, scale=1.5, rotate=(0.0, 45.0, 20.0), translate=(0.1, 0.1, 0.2))
    light = sb.add_material(Material.diffuse_light((12.0, 12.0, 12.0)))
    sb.add_light_quad((-0.75, 3.0, -0.75), (1.5, 0, 0), (0, 0, 1.5), light)
    sb.set_solid((0.05, 0.05, 0.08))
    return sb


def test_gpu_gem_trace_matches_oracle():
    sb = gem_field()
    g, o = GpuScene(sb), O.OracleScene(sb)
    rs = np.concatenate([random_rays(60000, 7, center=(0, 0.5, 0), radius=3.0, spread=0.8),
                         camera_rays(make_camera((0.0, 1.6, 4.0), (0.0, 0.4, 0.0), vfov=35.0, aspect=1.0), 128, 128)])
    gh, oh = g.trace_closest(rs), o.trace_closest(rs)
    assert (oh["prim"] >= 5).sum() > 2000           # many rays end on a gem (ids after the quads and sphere)
    assert_same_hits(gh, oh)
    assert np.array_equal(g.trace_any(rs), o.trace_any(rs))


def test_gpu_convex_known_answers():
    pl = np.array([[1, 0, 0, 1], [-1, 0, 0, 1], [0, 1, 0, 50], [0, -1, 0, 50], [0, 0, 1, 50], [0, 0, -1, 50]],
                  np.float32)
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_convex(pl, m, (-1, -50, -50), (1, 50, 50))
    sb.add_diamond((10.0, 0.0, 0.0), 1.0, sb.add_material(Material.dielectric(1.5)))
    g = GpuScene(sb)
    h = g.trace_closest(rays(ray((-5, 0, 0), (1, 0, 0), 0.001, 4.0),
                             ray((-5, 0, 0), (1, 0, 0), 0.001, np.float32(4.0) - np.float32(1e-4)),
                             ray((10, 10, 0), (0, -1, 0), 0.001, 100.0),
                             ray((10, 0.3, 0), (1, 0, 0), 0.001, 100.0)))
    assert h["prim"][0] == 0 and abs(h["t"][0] - 4.0) < 1e-6 and h["prim"][1] == -1
    assert h["prim"][2] == 1 and h["b1"][2:3].view(np.int32)[0] == 0        # the table plane from above
    assert h["prim"][3] == 1                                                  # interior ray exits


@pytest.mark.parametrize("hero", [1, 4])
def test_gpu_gem_render_matches_oracle(hero):
    sb = gem_field()
    sb.spectral_range = 1 if hero > 1 else 0
    cam = make_camera((0.0, 1.6, 4.0), (0.0, 0.4, 0.0), vfov=35.0, aspect=1.0)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = pass_params(64, 64, 0, 64, 8, 12, hero, 1.0, 31)
    gi = g.render_pass(cam, p)
    p.seed = 32
    oi = o.render_pass(cam, p)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)


def test_gpu_toml_gem_sun_caustics_match_oracle():
    doc = {"camera": {"look_from": [0, 0.02, -0.03], "look_at": [0, 0, 0]},
           "background": {"type": "physical", "sun_elevation": 60.0, "sun_azimuth": 20.0},
           "objects": [{"shape": {"type": "quad", "corner": [-0.05, -0.004, -0.05], "u": [0.1, 0, 0],
                                  "v": [0, 0, 0.1]}, "material": {"type": "lambertian", "color": [0.8, 0.8, 0.8]}}],
           "gems": [{"carat": 1.0, "center": [0, 0.001, 0], "color_grade": "H", "rotate": [5.0, 0.0, 0.0],
                     "spin": 15.0},
                    {"measurements_mm": [8.99, 6.42, 3.97], "table_pct": 58.0, "crown_pct": 16.0,
                     "pavilion_pct": 41.0, "material": "sapphire", "center": [0.012, 0.001, 0.004]}]}
    sb = scene_from_toml_dict(doc)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = photons.caustic_params(sb, 1000000, 0.002, seed=5)
    ng, no = g.photon_build(p), o.photon_build(p)
    assert ng > 200 and abs(ng - no) <= max(30, no // 20), (ng, no)
    gp, gw, _, gi = g.photon_export()
    op, ow, _, oi = o.photon_export()
    common, ga, oa = np.intersect1d(gi, oi, return_indices=True)
    assert len(common) > 0.95 * min(ng, no)
    np.testing.assert_allclose(gw[ga], ow[oa], rtol=1e-3, atol=1e-7)


def step_field():
    """Step-family cuts (princess with chevrons, cushion, trillion, a 626-plane
    marquise, an emerald step cut) and a round brilliant, as [[gems]] entries."""
    gems = [dict(measurements_mm=[6.0, 5.9, 4.2], table_pct=65.0, crown_pct=12.0, pavilion_pct=50.0, cut="princess",
                 material="sapphire", rotate_y=25.0, center=[-1.2, 0.45, 0.3], scale_mm=0.3),
            dict(measurements_mm=[6.0, 6.0, 3.7], cut="brilliant", material="diamond", center=[0.0, 0.45, 0.0],
                 scale_mm=0.3),
            dict(measurements_mm=[6.0, 5.0, 3.5], cut="cushion", material="ruby", center=[1.2, 0.45, 0.3],
                 scale_mm=0.3, rotate=[0.0, 0.0, 15.0]),
            dict(measurements_mm=[6.0, 6.0, 3.5], cut="trillion", material="emerald", center=[-0.6, 0.35, -1.0],
                 scale_mm=0.3),
            dict(measurements_mm=[9.0, 4.0, 3.0], cut="marquise", center=[0.7, 0.3, -1.0], scale_mm=0.3,
                 spin=40.0),
            dict(measurements_mm=[8.0, 6.0, 4.0], cut="step", material="emerald", center=[0.0, 0.4, 1.2],
                 scale_mm=0.3, polish=0.05)]
    doc = {"camera": {"look_from": [0.0, 2.0, 4.0], "look_at": [0.0, 0.3, 0.0]},
           "background": {"type": "physical", "sun_elevation": 25.0, "sun_azimuth": 30.0},
           "objects": [{"shape": {"type": "quad", "corner": [-4, 0, -4], "u": [8, 0, 0], "v": [0, 0, 8]},
                        "material": {"type": "checker", "even": [0.1, 0.1, 0.1], "odd": [0.8, 0.8, 0.8],
                                     "scale": 0.5}}],
           "lights": [{"corner": [-0.75, 3.0, -0.75], "u": [1.5, 0, 0], "v": [0, 0, 1.5], "temp_k": 6500.0,
                       "intensity": 8.0}],
           "gems": gems}
    return scene_from_toml_dict(doc)


def test_gpu_step_cut_trace_matches_oracle():
    sb = step_field()
    assert max(len(c["planes"]) for c in sb.convex) == 626
    g, o = GpuScene(sb), O.OracleScene(sb)
    rs = np.concatenate([random_rays(60000, 11, center=(0, 0.4, 0), radius=3.0, spread=0.8),
                         camera_rays(make_camera((0.0, 2.0, 4.0), (0.0, 0.3, 0.0), vfov=35.0, aspect=1.0), 128, 128)])
    gh, oh = g.trace_closest(rs), o.trace_closest(rs)
    assert (oh["prim"] >= 2).sum() > 2000
    assert_same_hits(gh, oh)
    assert np.array_equal(g.trace_any(rs), o.trace_any(rs))


def test_gpu_step_cut_render_matches_oracle():
    sb = step_field()
    sb.spectral_range = 1
    cam = make_camera((0.0, 2.0, 4.0), (0.0, 0.3, 0.0), vfov=35.0, aspect=1.0)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = pass_params(64, 64, 0, 64, 8, 12, 4, 1.0, 41)
    gi = g.render_pass(cam, p)
    p.seed = 42
    oi = o.render_pass(cam, p)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)


def test_gpu_interior_rays_in_overlapping_gems_match_oracle():
    """Rays that start inside two overlapping stones (as refracted and
    internally reflected rays do) end on the nearer exit on both paths."""
    sb = step_field()
    rng = np.random.default_rng(8)
    lo = np.array([min(c["pivot"][a] for c in sb.convex) - 0.6 for a in range(3)])
    hi = np.array([max(c["pivot"][a] for c in sb.convex) + 0.6 for a in range(3)])
    n = 100000
    o = lo + (hi - lo) * rng.random((n, 3))
    d = rng.normal(0, 1, (n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rs = np.concatenate([o, d, np.full((n, 1), 0.001), np.full((n, 1), np.inf)], 1).astype(np.float32)
    g, orc = GpuScene(sb), O.OracleScene(sb)
    gh, oh = g.trace_closest(rs), orc.trace_closest(rs)
    assert (oh["prim"] >= 2).sum() > n // 4
    assert_same_hits(gh, oh)
    assert np.array_equal(g.trace_any(rs), orc.trace_any(rs))


def test_gpu_gem_room_matches_oracle():
    """The reference's benchmark room (bench.toml layout: gems, PBR ball,
    blackbody panel, dusk sky, caustic photon map) at a reduced size."""
    from rustracer_b200 import configs
    sb, st = configs.gem_room_scene(width=96, height=64)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = photons.caustic_params(sb, st["photons"], st["radius"], seed=1)
    ng, no = g.photon_build(p), o.photon_build(p)
    assert ng > 1000 and abs(ng - no) <= max(30, no // 20), (ng, no)
    pp = pass_params(96, 64, 0, 64, 8, 16, 1, 1.0, 81)
    gi = g.render_pass(st["camera"], pp)
    pp.seed = 82
    oi = o.render_pass(st["camera"], pp)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)
