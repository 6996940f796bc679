"""Textures on the GPU against the CPU oracle: image and mottle Lambertian
albedos, a textured PBR mesh (albedo, roughness, metallic, ambient occlusion
and normal maps through the mesh tangents) and the default triangle UVs;
render tiles within 3 SE."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.renderer import GpuScene, pass_params
from rustracer_b200.scene import Material, SceneBuilder, make_camera
from tests.test_gpu_render import assert_tiles_agree

pytestmark = pytest.mark.gpu


def uv_sphere(center, r, nu=48, nv=24):
    """A latitude-longitude sphere mesh with per-vertex UVs."""
    V, UV, F = [], [], []
    for j in range(nv + 1):
        th = math.pi * j / nv
        for i in range(nu + 1):
            ph = 2 * math.pi * i / nu
            V.append([center[0] + r * math.sin(th) * math.cos(ph), center[1] + r * math.cos(th),
                      center[2] + r * math.sin(th) * math.sin(ph)])
            UV.append([i / nu, 1.0 - j / nv])
    for j in range(nv):
        for i in range(nu):
            a, b = j * (nu + 1) + i, j * (nu + 1) + i + 1
            c, d = a + nu + 1, b + nu + 1
            F += [[a, c, b], [b, c, d]]
    return np.array(V), np.array(F), np.array(UV)


def texture_scene():
    rng = np.random.default_rng(3)
    sb = SceneBuilder()
    checker = np.zeros((64, 64, 3), np.uint8)
    checker[(np.arange(64)[:, None] // 8 + np.arange(64)[None, :] // 8) % 2 == 0] = (220, 200, 170)
    checker[(np.arange(64)[:, None] // 8 + np.arange(64)[None, :] // 8) % 2 == 1] = (40, 60, 90)
    floor = Material.lambertian((0, 0, 0))
    floor.albedo_tex = sb.add_texture_image(checker)
    sb.add_quad((-4, 0, -4), (8, 0, 0), (0, 0, 8), sb.add_material(floor))
    mottle = Material.lambertian((0, 0, 0))
    mottle.albedo_tex = sb.add_texture_mottle((0.2, 0.5, 0.3), (0.8, 0.7, 0.2), 4.0)
    sb.add_sphere((-1.3, 0.5, 0.0), 0.5, sb.add_material(mottle))
    # textured PBR on a UV-mapped mesh
    alb = (rng.random((32, 64, 3)) * 255).astype(np.uint8)
    rough = np.repeat((np.linspace(0.1, 0.9, 64)[None, :, None] * 255).astype(np.uint8), 32, 0).repeat(3, 2)
    metal = np.zeros((32, 64, 3), np.uint8)
    metal[:, 32:] = 255
    ao = np.full((32, 64, 3), 200, np.uint8)
    nrm = np.empty((32, 64, 3), np.uint8)
    tilt = rng.normal(0, 0.25, (32, 64, 2))
    nz = np.sqrt(np.clip(1 - (tilt ** 2).sum(-1), 0, 1))
    nrm[..., 0], nrm[..., 1] = ((tilt[..., 0] + 1) * 127.5).astype(np.uint8), ((tilt[..., 1] + 1) * 127.5).astype(np.uint8)
    nrm[..., 2] = ((nz + 1) * 127.5).astype(np.uint8)
    pbr = Material.pbr((0.8, 0.8, 0.8), roughness=0.5, metallic=0.0)
    pbr.albedo_tex, pbr.roughness_tex = sb.add_texture_image(alb), sb.add_texture_image(rough)
    pbr.metallic_tex, pbr.ao_tex = sb.add_texture_image(metal), sb.add_texture_image(ao)
    pbr.normal_tex = sb.add_texture_image(nrm)
    V, F, UV = uv_sphere((0.0, 0.6, -0.2), 0.6)
    sb.add_mesh(V, F, sb.add_material(pbr), uvs=UV)
    # a mesh without UVs sampling an image (mesh.rs's default corner UVs)
    img = Material.lambertian((0, 0, 0))
    img.albedo_tex = sb.add_texture_image(alb)
    V2 = np.array([[1.0, 0.0, -0.5], [2.0, 0.0, -0.5], [1.5, 1.2, -0.2]])
    sb.add_mesh(V2, np.array([[0, 1, 2]]), sb.add_material(img))
    light = sb.add_material(Material.diffuse_light((8.0, 8.0, 8.0)))
    sb.add_light_quad((-0.75, 3.0, -0.75), (1.5, 0, 0), (0, 0, 1.5), light)
    sb.set_physical(35.0, 40.0, 3.0)
    return sb


@pytest.mark.parametrize("hero", [1, 4])
def test_gpu_texture_render_matches_oracle(hero):
    sb = texture_scene()
    sb.spectral_range = 1 if hero > 1 else 0
    cam = make_camera((0.0, 1.6, 3.8), (0.0, 0.5, 0.0), vfov=40.0, aspect=1.0)
    g, o = GpuScene(sb), O.OracleScene(sb)
    p = pass_params(64, 64, 0, 64, 8, 8, hero, 1.0, 71)
    gi = g.render_pass(cam, p)
    p.seed = 72
    oi = o.render_pass(cam, p)
    assert np.isfinite(gi).all()
    assert_tiles_agree(gi, oi)
