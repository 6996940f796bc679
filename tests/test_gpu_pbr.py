"""PbrMaterial on the GPU against the CPU oracle: anisotropic metal,
clearcoat with a thin film, sheen, an emissive PBR light in the NEE list, the
specular sun NEE of the PBR lobes, and caustic photons off a PBR conductor
stored on a PBR floor."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200 import photons
from rustracer_b200.renderer import GpuScene, pass_params
from rustracer_b200.scene import Material, SceneBuilder, make_camera
from tests.test_gpu_render import assert_tiles_agree

pytestmark = pytest.mark.gpu


def pbr_scene(sky=True):
    sb = SceneBuilder()
    floor = sb.add_material(Material.pbr((0.6, 0.6, 0.55), roughness=0.8))
    gold = sb.add_material(Material.pbr((1.0, 0.78, 0.34), roughness=0.25, metallic=1.0, anisotropy=0.7,
                                        anisotropy_angle=0.5))
    paint = sb.add_material(Material.pbr((0.1, 0.25, 0.6), roughness=0.4, clearcoat=1.0, clearcoat_roughness=0.05,
                                         film_thickness=450.0, film_ior=1.4))
    cloth = sb.add_material(Material.pbr((0.6, 0.1, 0.15), roughness=0.9, sheen=1.0, sheen_tint=0.7))
    glow = sb.add_material(Material.pbr((0.2, 0.2, 0.2), emission=(1.0, 0.7, 0.4), emission_strength=6.0))
    sb.add_quad((-4, 0, -4), (8, 0, 0), (0, 0, 8), floor)
    sb.add_sphere((-1.1, 0.5, 0.0), 0.5, gold)
    sb.add_sphere((0.0, 0.5, -0.3), 0.5, paint)
    sb.add_sphere((1.1, 0.5, 0.0), 0.5, cloth)
    sb.add_light_quad((-0.5, 2.5, -0.5), (1.0, 0, 0), (0, 0, 1.0), glow)
    if sky:
        sb.set_physical(30.0, 35.0, 3.0)
    else:
        sb.set_solid((0.2, 0.25, 0.3))
    return sb


@pytest.mark.parametrize("hero,sky", [(1, True), (4, True), (1, False)])
def test_gpu_pbr_render_matches_oracle(hero, sky):
    sb = pbr_scene(sky)
    sb.spectral_range = 1 if hero > 1 else 0
    cam = make_camera((0.0, 1.4, 3.6), (0.0, 0.45, 0.0), vfov=40.0, aspect=1.0)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = pass_params(64, 64, 0, 64, 8, 8, hero, 1.0, 51)
    gi = g.render_pass(cam, p)
    p.seed = 52
    oi = o.render_pass(cam, p)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)


def test_gpu_pbr_sun_photons_match_oracle():
    sb = pbr_scene(True)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = photons.caustic_params(sb, 400000, 0.05, seed=9)
    ng, no = g.photon_build(p), o.photon_build(p)
    assert ng > 200 and abs(ng - no) <= max(30, no // 20), (ng, no)
    gp, gw, _, gi = g.photon_export()
    op, ow, _, oi = o.photon_export()
    common, ga, oa = np.intersect1d(gi, oi, return_indices=True)
    assert len(common) > 0.95 * min(ng, no)
    # the same photons carry the same power, up to a few whose grazing GGX
    # bounces amplify the last-ulp differences of the device math functions
    close = np.isclose(gw[ga], ow[oa], rtol=1e-3, atol=1e-7).all(1)
    assert close.mean() > 0.995, close.mean()
    np.testing.assert_allclose(gw[ga].sum(0), ow[oa].sum(0), rtol=2e-3)
