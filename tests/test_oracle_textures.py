"""Textures in the CPU oracle: Texture::value (texture.rs:25-57, pinned to
its mottle test texture.rs:65-79), the PBR bilinear samplers
(material.rs:633-671), hit UVs and tangents (triangle.rs:91-107, mesh.rs:33-81,
quad.rs:53-56, sphere.rs:11-15), and the TOML texture materials."""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.output import write_png
from rustracer_b200.scene import Material, SceneBuilder, load_obj, mesh_tangents, scene_from_toml_dict
from tests.helpers import ray, rays


def _srgb(c):
    v = np.float32(c) / np.float32(255.0)
    return v / 12.92 if v <= 0.04045 else ((v + 0.055) / 1.055) ** 2.4


def _tex_scene(img=None, mottle=None):
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_sphere((0, 0, 0), 1.0, m)
    tid = sb.add_texture_image(img) if img is not None else sb.add_texture_mottle(*mottle)
    return sb, tid


def test_mottle_stays_within_lo_hi():
    lo, hi = (0.40, 0.40, 0.42), (0.45, 0.45, 0.47)
    sb, tid = _tex_scene(mottle=(lo, hi, 3.0))
    i = np.arange(2000, dtype=np.float32)
    p = np.stack([i * np.float32(0.371), np.zeros_like(i), i * np.float32(0.113)], 1)
    c = O.OracleScene(sb).tex_sample(tid, np.zeros((2000, 2)), p)
    assert (c >= np.minimum(lo, hi) - 1e-6).all() and (c <= np.maximum(lo, hi) + 1e-6).all()
    assert c[:, 0].std() > 1e-3                                       # it does vary


def test_image_value_is_the_nearest_texel_srgb_decoded():
    img = np.array([[[10, 20, 30], [200, 100, 50]], [[0, 255, 128], [64, 64, 64]]], np.uint8)
    sb, tid = _tex_scene(img=img)
    s = O.OracleScene(sb)
    # u → column, 1 − v → row (v = 1 is the top row)
    c = s.tex_sample(tid, [[0.1, 0.9], [0.9, 0.9], [0.1, 0.1], [0.9, 0.1], [1.5, -2.0]])
    want = [img[0, 0], img[0, 1], img[1, 0], img[1, 1], img[1, 1]]
    for k in range(5):
        np.testing.assert_allclose(c[k], [_srgb(x) for x in want[k]], rtol=1e-6)


def test_bilinear_samplers():
    img = np.array([[[0, 0, 0], [255, 255, 255]]], np.uint8)       # 1 × 2: black | white
    sb, tid = _tex_scene(img=img)
    s = O.OracleScene(sb)
    # texel centres at u = 0.25, 0.75; u = 0.5 is half way
    raw = s.tex_sample(tid, [[0.25, 0.5], [0.5, 0.5], [0.75, 0.5], [0.0, 0.5]], mode=1)
    np.testing.assert_allclose(raw[:, 0], [0.0, 0.5, 1.0, 0.0], atol=1e-6)
    lin = s.tex_sample(tid, [[0.5, 0.5]], mode=2)
    assert abs(lin[0, 0] - 0.5) < 1e-6
    srgb = s.tex_sample(tid, [[0.5, 0.5]], mode=0)                   # decode first, then blend
    assert abs(srgb[0, 0] - 0.5) < 1e-6


def test_hit_uvs_and_tangents():
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    # a triangle without texcoords: mesh.rs's (0,0) (1,0) (0.5,1) and a (1,0,0) tangent
    sb.add_mesh(np.array([[0, 0, 0], [2, 0, 0], [0, 2, 0]], float), np.array([[0, 1, 2]]), m)
    # a triangle with texcoords and a derived tangent
    V = np.array([[0, 0, 5], [2, 0, 5], [0, 2, 5]], float)
    sb.add_mesh(V, np.array([[0, 1, 2]]), m, uvs=np.array([[0.0, 0.0], [0.0, 1.0], [1.0, 0.0]]))
    sb.add_quad((10, 0, 0), (1, 0, 0), (0, 1, 0), m)
    sb.add_sphere((0, 0, -10), 1.0, m)
    s = O.OracleScene(sb)
    r = s.hit_uv(rays(ray((0.5, 0.5, -1), (0, 0, 1)), ray((0.5, 0.5, 4), (0, 0, 1)), ray((10.25, 0.75, 1), (0, 0, -1)),
                      ray((0, 0, -20), (0, 0, 1))))
    b1, b2 = 0.25, 0.25                                               # (0.5, 0.5) in the 2 × 2 triangle
    assert abs(r[0, 0] - (b1 + 0.5 * b2)) < 1e-6 and abs(r[0, 1] - b2) < 1e-6
    np.testing.assert_allclose(r[0, 2:], [1, 0, 0], atol=1e-6)
    assert abs(r[1, 0] - b2) < 1e-6 and abs(r[1, 1] - b1) < 1e-6    # u along the y edge, v along x
    np.testing.assert_allclose(r[1, 2:], [0, 1, 0], atol=1e-6)       # dP/du = +y
    assert abs(r[2, 0] - 0.25) < 1e-6 and abs(r[2, 1] - 0.75) < 1e-6 # quad (α, β)
    # sphere: the hit point (0, 0, -11) has outward normal (0, 0, -1): φ = atan2(1, 0) + π, θ = π/2
    assert abs(r[3, 0] - (math.pi / 2 + math.pi) / (2 * math.pi)) < 1e-6 and abs(r[3, 1] - 0.5) < 1e-6


def test_mesh_tangents_follow_the_uv_gradient():
    V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    F = np.array([[0, 1, 2], [0, 2, 3]])
    T = mesh_tangents(V, F, np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32))
    np.testing.assert_allclose(T, np.tile([1, 0, 0], (4, 1)), atol=1e-6)
    T2 = mesh_tangents(V, F, np.zeros((4, 2), np.float32))           # degenerate UVs: the (1,0,0) fallback
    np.testing.assert_allclose(T2, np.tile([1, 0, 0], (4, 1)))


def test_obj_texcoords_single_index(tmp_path):
    p = tmp_path / "q.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvt 1 0\nvt 1 1\nvt 0 1\nf 1/1 2/2 3/3 4/4\n")
    V, F, N, UV = load_obj(str(p), with_uv=True)
    assert len(V) == 4 and F.shape == (2, 3) and N is None
    np.testing.assert_allclose(UV[F[0]], [[0, 0], [1, 0], [1, 1]])


def test_texture_materials_from_toml(tmp_path):
    img = (np.random.default_rng(0).random((8, 8, 3)) * 255).astype(np.uint8)
    write_png(str(tmp_path / "a.png"), img)
    doc = {"camera": {"look_from": [0, 0, -5], "look_at": [0, 0, 0]},
           "objects": [{"shape": {"type": "sphere", "center": [0, 0, 0], "radius": 1.0},
                        "material": {"type": "image", "path": "a.png"}},
                       {"shape": {"type": "sphere", "center": [3, 0, 0], "radius": 1.0},
                        "material": {"type": "noise", "lo": [0.4, 0.4, 0.42], "hi": [0.45, 0.45, 0.47]}},
                       {"shape": {"type": "sphere", "center": [6, 0, 0], "radius": 1.0},
                        "material": {"type": "metal", "color": [0.9, 0.8, 0.7], "fuzz": 0.1}},
                       {"shape": {"type": "sphere", "center": [9, 0, 0], "radius": 1.0},
                        "material": {"type": "textured_pbr", "albedo_path": "a.png", "roughness_path": "a.png",
                                     "normal_path": "a.png"}}]}
    sb = scene_from_toml_dict(doc, str(tmp_path))
    mats = sb.materials
    assert mats[0].albedo_tex == 1 and mats[1].albedo_tex == 2 and mats[1].type == 0
    assert mats[2].type == 7 and mats[2].metallic == 1.0 and abs(mats[2].roughness - 0.1) < 1e-7
    assert mats[3].albedo_tex == 3 and mats[3].roughness_tex == 4 and mats[3].normal_tex == 5
    assert mats[3].metallic_tex == 0 and mats[3].ao_tex == 0
    s = O.OracleScene(sb)
    np.testing.assert_allclose(s.tex_sample(1, [[0.01, 0.99]]), [[_srgb(x) for x in img[0, 0]]], rtol=1e-6)


def _rgbe(c):
    """float RGB → RGBE bytes (the Radiance encoding)."""
    m = max(c)
    if m < 1e-32:
        return [0, 0, 0, 0]
    f, e = math.frexp(m)
    sc = f * 256.0 / m
    return [int(c[0] * sc), int(c[1] * sc), int(c[2] * sc), e + 128]


def test_radiance_hdr_flat_and_rle_scanlines(tmp_path):
    """load_hdr's scanline decoder (native rt_rgbe_decode): one flat row and
    one new-style RLE row with a run and a literal block, width ≥ 256 so the
    width field needs both bytes."""
    from rustracer_b200.scene import load_hdr
    W = 300
    rng = np.random.default_rng(1)
    row0 = [_rgbe(rng.random(3) * 4) for _ in range(W)]
    row1 = [_rgbe((0.5, 0.25, 0.125))] * 200 + [_rgbe(rng.random(3)) for _ in range(W - 200)]
    body = bytearray(b"".join(bytes(px) for px in row0))
    body += bytes([2, 2, W >> 8, W & 255])
    for c in range(4):
        ch = [px[c] for px in row1]
        x = 0
        while x < W:
            if x < 200:                                  # runs of ≤ 127
                n = min(127, 200 - x)
                body += bytes([128 + n, ch[x]])
            else:                                        # literals of ≤ 128
                n = min(128, W - x)
                body += bytes([n] + ch[x:x + n])
            x += n
    p = tmp_path / "t.hdr"
    p.write_bytes(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 2 +X %d\n" % W + bytes(body))
    img = load_hdr(str(p))
    want = np.array([[[q[k] * math.ldexp(1.0, q[3] - 136) if q[3] else 0.0 for k in range(3)] for q in r]
                     for r in (row0, row1)], np.float32)
    np.testing.assert_array_equal(img, want)
