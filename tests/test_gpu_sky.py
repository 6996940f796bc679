"""Physical (Preetham) sky on the GPU against the CPU oracle: sun NEE at
diffuse vertices and at rough conductors, the sun-disc MIS weights on escaped
rays, and the sun as the caustic photon source."""
import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200 import photons
from rustracer_b200.renderer import GpuScene, pass_params
from rustracer_b200.scene import Material, make_camera
from tests.helpers import physical_sky_scene
from tests.test_gpu_render import assert_tiles_agree

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("hero,roughness", [(1, 0.3), (4, 0.15)])
def test_gpu_physical_sky_render_matches_oracle(hero, roughness):
    sb = physical_sky_scene(elevation=35.0, azimuth=30.0, roughness=roughness)
    sb.spectral_range = 1 if hero > 1 else 0
    cam = make_camera((0.0, 1.2, 3.5), (0.0, 0.4, 0.0), vfov=40.0, aspect=1.0)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = pass_params(64, 64, 0, 64, 8, 8, hero, 1.0, 21)
    gi = g.render_pass(cam, p)
    p.seed = 22
    oi = o.render_pass(cam, p)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)


def test_gpu_sun_photons_match_oracle():
    sb = physical_sky_scene(elevation=50.0)
    glass = sb.add_material(Material.spectral_dielectric_cauchy(1.5, 0.0042))
    sb.add_sphere((0.0, 1.3, 0.6), 0.3, glass)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = photons.caustic_params(sb, 400000, 0.05, seed=3)
    assert p.emitters[0].type == photons.abi.RT_EMIT_SUN
    ng, no = g.photon_build(p), o.photon_build(p)
    assert ng > 200 and abs(ng - no) <= max(30, no // 20), (ng, no)
    gp, gw, _, gi = g.photon_export()
    op, ow, _, oi = o.photon_export()
    common, ga, oa = np.intersect1d(gi, oi, return_indices=True)
    assert len(common) > 0.95 * min(ng, no)
    np.testing.assert_allclose(gw[ga], ow[oa], rtol=1e-3, atol=1e-7)


def test_gpu_sun_emitter_needs_physical_sky():
    from tests.helpers import unit_quad_scene
    g = GpuScene(unit_quad_scene())
    with pytest.raises(Exception):
        g.photon_build(photons.photon_params([photons.sun_emitter(1000)], 0.1))
