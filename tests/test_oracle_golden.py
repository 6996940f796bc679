"""Pins the CPU oracle against the known-answer tests of the reference's own
unit tests (cited per test).  No GPU needed."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.scene import Material, SceneBuilder
from tests.helpers import ray, rays, spheres_scene, unit_quad_scene, xy_triangle_scene


# ── quad.rs:129-198 ──────────────────────────────────────────────────────────
def test_quad_hits_and_misses():
    s = O.OracleScene(unit_quad_scene())
    h = s.trace_closest(rays(
        ray((0.5, 0.5, 3.0), (0, 0, -1)),      # quad.rs:130-135  t = 3
        ray((0.25, 0.75, 1.0), (0, 0, -1)),    # quad.rs:150-155  uv = (0.25, 0.75)
        ray((0, 0, 1), (0, 0, -1)), ray((1, 0, 1), (0, 0, -1)), ray((0, 1, 1), (0, 0, -1)), ray((1, 1, 1), (0, 0, -1)),
        ray((1.01, 0.5, 1.0), (0, 0, -1)),     # quad.rs:168-171 miss outside u
        ray((0.5, -0.01, 1.0), (0, 0, -1)),    # quad.rs:174-177 miss outside v
        ray((0.5, 0.5, 0.0), (1, 0, 0)),       # quad.rs:180-184 parallel
    ))
    assert abs(h["t"][0] - 3.0) < 1e-5
    assert abs(h["b1"][1] - 0.25) < 1e-5 and abs(h["b2"][1] - 0.75) < 1e-5
    assert (h["prim"][2:6] == 0).all()         # closed corners (quad.rs:158-165)
    assert (h["prim"][6:] == -1).all()


def test_degenerate_quad_is_rejected():
    # quad.rs:137-147: the reference panics; the C ABI reports RT_ERR_INVALID
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((1, 1, 1)))
    sb.add_quad((0, 0, 0), (1, 0, 0), (2, 0, 0), m)
    with pytest.raises(ValueError, match="degenerate"):
        O.OracleScene(sb)


# ── triangle.rs:245-311 ──────────────────────────────────────────────────────
def test_triangle_known_answers():
    s = O.OracleScene(xy_triangle_scene())
    h = s.trace_closest(rays(
        ray((2 / 3, 2 / 3, -5.0), (0, 0, 1)),  # :246-252 centroid t = 5
        ray((0.0, 0.0, -3.0), (0, 0, 1)),      # :255-260 vertex t = 3
        ray((3.0, 0.0, -1.0), (0, 0, 1)),      # :263-267 b1 > 1
        ray((0.0, -1.0, -1.0), (0, 0, 1)),     # :270-274 b2 < 0
        ray((1.5, 1.5, -1.0), (0, 0, 1)),      # :277-281 b1 + b2 > 1
        ray((0.5, 0.5, 0.0), (1, 0, 0)),       # :284-288 parallel
        ray((2 / 3, 2 / 3, -1.0), (0, 0, 1)),  # :291-311 barycentric (1/3, 1/3)
    ))
    assert abs(h["t"][0] - 5.0) < 1e-5
    assert abs(h["t"][1] - 3.0) < 1e-5
    assert (h["prim"][2:6] == -1).all()
    assert abs(h["b1"][6] - 1 / 3) < 1e-5 and abs(h["b2"][6] - 1 / 3) < 1e-5


# ── sphere.rs:132-138, bvh.rs:684-745 ────────────────────────────────────────
def test_sphere_zero_direction_misses():
    s = O.OracleScene(spheres_scene([(0, 0, 0)]))
    h = s.trace_closest(rays(ray((0, 0, -5), (0, 0, 0))))
    assert h["prim"][0] == -1
    assert s.trace_any(rays(ray((0, 0, -5), (0, 0, 0))))[0] == 0


def test_bvh_sphere_cases():
    s = O.OracleScene(spheres_scene([(0, 0, 0)]))
    assert s.trace_closest(rays(ray((0, 0, -5), (0, 0, 1))))["prim"][0] == 0          # :685-691
    assert s.trace_closest(rays(ray((2, 0, -5), (0, 0, 1))))["prim"][0] == -1         # :694-701
    occ = s.trace_any(rays(ray((0, 0, -5), (0, 0, 1)), ray((2, 0, -5), (0, 0, 1))))  # :704-712
    assert list(occ) == [1, 0]
    two = O.OracleScene(spheres_scene([(0, 0, -3), (0, 0, 3)]))                        # :715-725
    assert two.trace_closest(rays(ray((0, 0, -10), (0, 0, 1))))["t"][0] < 8.0
    pos = [(x * 10.0, y * 10.0, 0.0) for x in (-1, 0, 1) for y in (-1, 0, 1)]          # :728-745
    grid = O.OracleScene(spheres_scene(pos))
    h = grid.trace_closest(rays(*[ray((p[0], p[1], -20.0), (0, 0, 1)) for p in pos]))
    assert (h["prim"] >= 0).all()


def test_bvh_matches_brute_force():
    from tests.helpers import random_rays
    from rustracer_b200.configs import icosphere, vertex_normals
    V, F = icosphere(4)
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_mesh(V, F, m, vertex_normals(V, F))
    sb.add_quad((-2, -1.05, -2), (0, 0, 4), (4, 0, 0), m)
    sb.add_sphere((0.5, 1.2, 0.0), 0.3, m)
    s = O.OracleScene(sb)
    r = random_rays(20000, 3)
    a, b = s.trace_closest(r), s.trace_closest(r, brute=True)
    assert (a["prim"] == b["prim"]).all()
    assert np.array_equal(a["t"].view(np.uint32), b["t"].view(np.uint32))


# ── material.rs:1622-1639 (Fresnel), :1299-1436 (GGX) ─────────────────────────
def test_fresnel_dielectric():
    f = lambda c, e: O.scalar("fresnel_dielectric", c, e)
    assert abs(f(1.0, 1 / 1.5) - 0.04) < 1e-6 and abs(f(1.0, 1.5) - 0.04) < 1e-6
    assert abs(f(0.0, 1 / 1.5) - 1.0) < 1e-6
    assert f(0.5, 1.5) == 1.0
    c = lambda deg: math.cos(math.radians(deg))
    assert f(c(30), 1 / 1.5) < f(c(60), 1 / 1.5) < f(c(85), 1 / 1.5)


def test_ggx_ndf_integrates_to_one():
    for alpha in (0.1, 0.3, 0.7, 1.0):
        n = 1000
        dth = math.pi / 2 / n
        tot = sum(O.scalar("ggx_ndf", math.cos((i + 0.5) * dth), alpha) * math.cos((i + 0.5) * dth)
                  * math.sin((i + 0.5) * dth) * dth * 2 * math.pi for i in range(n))
        assert abs(tot - 1.0) < 0.01


def test_smith_terms():
    for alpha in (0.01, 0.1, 0.3, 0.5, 0.8, 1.0):
        for c in (0.01, 0.1, 0.3, 0.5, 0.7, 0.9, 1.0):
            g = O.scalar("smith_g1", c, alpha)
            assert 0.0 <= g <= 1.0
    for c in (0.1, 0.5, 0.9, 1.0):
        assert abs(O.scalar("smith_g1", c, 1e-6) - 1.0) < 1e-4
    for alpha in (0.01, 0.1, 0.5, 1.0):
        for c in (0.05, 0.3, 0.7, 1.0):
            lam, g1 = O.scalar("smith_lambda", c, alpha), O.scalar("smith_g1", c, alpha)
            assert abs(lam - (1 / g1 - 1)) < 1e-5
    for alpha in (0.05, 0.3, 1.0):                                      # material.rs:1408-1422
        for co in (0.2, 0.6, 1.0):
            for ci in (0.2, 0.6, 1.0):
                lo, li = O.scalar("smith_lambda", co, alpha), O.scalar("smith_lambda", ci, alpha)
                hc = 1 / (1 + lo + li)
                sep = O.scalar("smith_g1", co, alpha) * O.scalar("smith_g1", ci, alpha)
                assert sep - 1e-6 <= hc <= 1 + 1e-6


def test_e_lut_bounds():
    for mu in (0.02, 0.25, 0.5, 0.9, 1.0):
        for alpha in (0.01, 0.25, 0.7, 1.0):
            e = O.scalar("e_ss", mu, alpha)
            assert 0.0 < e <= 1.0 + 1e-4
            c = O.scalar("energy_comp", mu, alpha)
            assert 1.0 - 1e-6 <= c <= 10.0
    assert O.scalar("e_ss", 1.0, 0.001) > 0.99


# ── spectrum.rs:283-452 ──────────────────────────────────────────────────────
def test_spectrum_normalisation_and_hues():
    lams = [380.0 + 5 * i for i in range(65)]
    mean = np.mean([O.spectral_to_rgb(l) for l in lams], axis=0)
    assert np.all(np.abs(mean - 1.0) < 1e-4)
    fmean = np.mean([O.spectral_fire_rgb(l) for l in lams], axis=0)
    assert np.all(np.abs(fmean - 1.0) < 1e-4)
    lum = lambda c: 0.2126 * c[0] + 0.7152 * c[1] + 0.0722 * c[2]
    plain = lum(O.spectral_to_rgb(450)) / lum(O.spectral_to_rgb(550))
    fire = lum(O.spectral_fire_rgb(450)) / lum(O.spectral_fire_rgb(550))
    assert fire < plain * 0.8
    b, g, r = O.spectral_to_rgb(450), O.spectral_to_rgb(550), O.spectral_to_rgb(650)
    assert b[2] > b[0] and b[2] > b[1] and g[1] > g[0] and g[1] > g[2] and r[0] > r[1] and r[0] > r[2]
    fb, fg = O.spectral_fire_rgb(450), O.spectral_fire_rgb(550)
    assert fb[2] > fb[0] and fb[2] > fb[1] and fg[1] > fg[0] and fg[1] > fg[2]
    assert np.allclose(O.spectral_to_rgb(380), O.spectral_to_rgb(300), atol=1e-5)
    assert np.allclose(O.spectral_to_rgb(700), O.spectral_to_rgb(800), atol=1e-5)


def test_extended_range_normalisation():
    # 380–780 nm sampling: the 81-entry table is normalised to a white mean too
    lams = [380.0 + 5 * i for i in range(81)]
    mean = np.mean([O.spectral_to_rgb(l, range_mode=1) for l in lams], axis=0)
    assert np.all(np.abs(mean - 1.0) < 1e-4)


def test_planck_cauchy_conductor():
    p = lambda l, t: O.scalar("planck_raw", l, t)
    assert p(450, 6500) / p(650, 6500) > p(450, 3000) / p(650, 3000)
    assert p(550, 6000) > p(550, 3000) and p(550, 10000) > p(550, 6000)
    assert abs(O.scalar("cauchy_ior", 589.3, 1.507, 0.00375) - 1.52) < 0.005
    assert O.scalar("cauchy_ior", 450, 1.507, 0.00375) > O.scalar("cauchy_ior", 550, 1.507, 0.00375) > \
        O.scalar("cauchy_ior", 650, 1.507, 0.00375)
    assert O.scalar("fresnel_conductor", 0.001, 0.18, 3.0) > 0.99
    n, k = 0.23, 3.0
    want = ((n - 1) ** 2 + k * k) / ((n + 1) ** 2 + k * k)
    assert abs(O.scalar("fresnel_conductor", 1.0, n, k) - want) < 1e-4
    for c in (0.0, 0.1, 0.3, 0.5, 0.7, 0.9, 1.0):
        assert 0.0 <= O.scalar("fresnel_conductor", c, 1.5, 2.0) <= 1.0
    rb = O.scalar("fresnel_conductor", 1.0, *O.metal_ior(0, 440.0))
    rr = O.scalar("fresnel_conductor", 1.0, *O.metal_ior(0, 660.0))
    assert rb < 0.5 and rr > 0.9 and rr > 2 * rb
    rs = [O.scalar("fresnel_conductor", 1.0, *O.metal_ior(2, l)) for l in (450.0, 550.0, 650.0)]
    assert min(rs) > 0.9 and max(rs) - min(rs) < 0.06


def test_diamond_preset_dispersion():
    # scene_file.rs:1453-1468: diamond (B, C) = (2.351, 0.0230) gives nF - nC ≈ 0.044
    nf = O.scalar("cauchy_ior", 486.1, 2.351, 0.0230)
    nc = O.scalar("cauchy_ior", 656.3, 2.351, 0.0230)
    assert abs(nf - nc - 0.044) < 0.002


# ── renderer.rs:737-815 (env map) ────────────────────────────────────────────
def _env_scene(img, rot=0.0, visible=None):
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_sphere((0, -100, 0), 1.0, m)
    sb.set_env(img, rot, visible)
    return O.OracleScene(sb)


def test_env_bilinear_and_seam():
    img = np.zeros((2, 4, 3), np.float32)
    img[:, 2:] = 1.0
    s = _env_scene(img)
    assert abs(s.env_sample((0, 0, 1))[0] - 0.5) < 1e-6
    a = math.pi / 4
    assert abs(s.env_sample((math.sin(a), 0, math.cos(a)))[0] - 1.0) < 1e-6
    assert abs(s.env_sample((0, 0, -1))[0] - 0.5) < 1e-6
    a = 3 * math.pi / 4
    assert abs(s.env_sample((math.sin(a), 0, math.cos(a)))[0] - 1.0) < 1e-6


def test_env_rotation():
    img = np.zeros((4, 8, 3), np.float32)
    img[:, 1:3] = 5.0
    s = _env_scene(img, rot=90.0)
    assert s.env_sample((0, 0, 1))[0] > 4.0
    assert s.env_sample((-1, 0, 0))[0] < 1.0
    rng = np.random.default_rng(1)
    for _ in range(16):
        d, pdf = s.env_sample_dir(rng.random(4))
        d = d / np.linalg.norm(d)
        assert pdf > 0 and d[2] > abs(d[0])


def test_env_split_and_gradient():
    img = np.full((2, 4, 3), 2.0, np.float32)
    s = _env_scene(img, visible={"type": "solid", "color": (0.5, 0.5, 0.5)})
    assert abs(s.bg_eval((0, 1, 0))[0] - 0.5) < 1e-6
    assert abs(s.env_eval((0, 1, 0))[0] - 2.0) < 1e-6
    assert s.env_pdf((0, 1, 0)) > 0
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_sphere((0, -100, 0), 1.0, m)
    sb.set_gradient((1, 1, 1), (0.2, 0.2, 0.2))
    g = O.OracleScene(sb)
    assert abs(g.bg_eval((0, 1, 0))[0] - 1.0) < 1e-6 and abs(g.bg_eval((0, -1, 0))[0] - 0.2) < 1e-6


# ── main.rs:1253-1279 (firefly clamp) ────────────────────────────────────────
def test_firefly_clamp():
    acc = O.Accumulator(1)
    for _ in range(4):
        acc.add(np.zeros(3, np.float32), clamp=8.0, min_samples=4, floor=5.0)
    acc.add(np.full(3, 100.0, np.float32), clamp=8.0, min_samples=4, floor=5.0)
    assert abs(acc.acc[0, 0] / acc.n[0] - 1.0) < 1e-4
    acc = O.Accumulator(1)
    for _ in range(4):
        acc.add(np.zeros(3, np.float32), clamp=0.0)
    acc.add(np.full(3, 100.0, np.float32), clamp=0.0)
    assert abs(acc.acc[0, 0] / acc.n[0] - 20.0) < 1e-3


def test_non_finite_samples_dropped():
    acc = O.Accumulator(2)
    acc.add(np.array([[np.nan, 0, 0], [1, 1, 1]], np.float32))
    acc.add(np.array([[1, 1, 1], [np.inf, 1, 1]], np.float32))
    assert list(acc.n) == [1, 1] and np.all(np.isfinite(acc.acc))


# ── pdf.rs:356-411 ───────────────────────────────────────────────────────────
def test_light_pdf_is_area_solid_angle():
    # quad light pdf = d² / (|cos| · A) (quad.rs:82-89); unit quad seen head-on from 5 units
    sb = SceneBuilder()
    lm = sb.add_material(Material.diffuse_light((1, 1, 1)))
    sb.add_light_quad((0, 0, 0), (1, 0, 0), (0, 1, 0), lm)
    s = O.OracleScene(sb)
    pdf = s.lights_pdf_value((0.5, 0.5, -5.0), (0, 0, 1))
    assert abs(pdf - 25.0) < 1e-3
    assert s.lights_pdf_value((0.5, 0.5, -5.0), (0, 0, -1)) == 0.0
