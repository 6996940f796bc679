"""PbrMaterial in the CPU oracle (material.rs:680-1050): the white-furnace
tests of the reference (material.rs:1345-1470), and the consistency of the
sampled lobes with specular_brdf_cos / specular_sampling_pdf."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.scene import Material, scene_from_toml_dict

WO_N = ((0.0, 0.0, -1.0), (0.0, 0.0, -1.0))      # normal incidence: ray +z onto a -z normal


def _furnace(mat, n, seed):
    rng = np.random.default_rng(seed)
    wo, nn = WO_N
    lobe, att, _, _, _ = O.pbr_scatter(mat, np.tile(wo, (n, 1)), nn, rng.random((n, 4)))
    lum = att.astype(np.float64) @ np.array([0.2126, 0.7152, 0.0722])
    return float(np.where(lobe > 0, lum, 0.0).mean())


@pytest.mark.parametrize("roughness", [0.1, 0.5, 0.9])
def test_white_furnace_metallic_no_energy_gain(roughness):
    m = Material.pbr((1.0, 1.0, 1.0), roughness=roughness, metallic=1.0)
    mean = _furnace(m, 8000, 42)
    assert 0.85 < mean <= 1.05, mean


def test_rough_white_metal_recovers_energy_via_compensation():
    assert _furnace(Material.pbr((1.0, 1.0, 1.0), roughness=0.9, metallic=1.0), 20000, 7) > 0.9


def test_white_furnace_smooth_metallic_is_nearly_lossless():
    mean = _furnace(Material.pbr((1.0, 1.0, 1.0), roughness=0.05, metallic=1.0), 8000, 123)
    assert 0.95 < mean <= 1.05


def _rand_wo(rng, k, n):
    """k outgoing directions in the hemisphere of the unit normal n."""
    v = rng.normal(0, 1, (k, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v *= np.sign(v @ n)[:, None]
    return v


@pytest.mark.parametrize("aniso", [0.0, 0.8])
def test_base_lobe_weight_equals_brdf_over_pdf(aniso):
    """Without a clearcoat the sampled base-lobe weight F·(G2/G1)·comp/p_spec
    is specular_brdf_cos / specular_sampling_pdf at the sampled direction."""
    m = Material.pbr((0.9, 0.6, 0.3), roughness=0.4, metallic=0.7, anisotropy=aniso, anisotropy_angle=0.6)
    rng = np.random.default_rng(3)
    n = np.array([0.3, 0.8, -0.52])
    n /= np.linalg.norm(n)
    wo = _rand_wo(rng, 4000, n)
    xi = rng.random((4000, 4))
    lobe, att, d, bc, pdf = O.pbr_scatter(m, wo, n, xi)
    spec = (lobe == 1) & (pdf > 1e-3)
    assert spec.sum() > 1000
    np.testing.assert_allclose(att[spec], bc[spec] / pdf[spec][:, None], rtol=2e-3, atol=1e-5)


def test_specular_pdf_mass_matches_the_sampled_lobe_fraction():
    """∫ specular_sampling_pdf dω over the sphere = the probability that
    scatter returns a specular lobe (coat or base) above the horizon."""
    m = Material.pbr((0.5, 0.5, 0.5), roughness=0.5, metallic=0.2, clearcoat=0.8, clearcoat_roughness=0.2)
    rng = np.random.default_rng(11)
    n = np.array([0.0, 1.0, 0.0])
    wo = np.array([0.6, 0.8, 0.0])
    k = 400000
    wi = rng.normal(0, 1, (k, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    _, _, _, _, pdf = O.pbr_scatter(m, np.tile(wo, (k, 1)), n, rng.random((k, 4)), spec_wi=wi)
    mass = float(pdf.astype(np.float64).mean() * 4 * math.pi)
    lobe, _, _, _, _ = O.pbr_scatter(m, np.tile(wo, (k, 1)), n, rng.random((k, 4)))
    frac = float((lobe == 1).mean())
    assert abs(mass - frac) < 0.02, (mass, frac)


def test_diffuse_lobe_with_sheen_known_answer():
    """albedo·(1−m) + π·sheen·(1−m)·C_sheen·(1−cos_o)^5, over (1−p_spec)(1−p_coat)."""
    albedo, metallic, sheen, tint = np.array([0.5, 0.4, 0.2]), 0.25, 0.8, 0.5
    m = Material.pbr(tuple(albedo), roughness=0.5, metallic=metallic, sheen=sheen, sheen_tint=tint)
    n = np.array([0.0, 1.0, 0.0])
    wo = np.array([math.sqrt(0.75), 0.5, 0.0])
    lobe, att, _, _, _ = O.pbr_scatter(m, wo[None], n, np.array([[0.5, 0.999, 0.3, 0.3]]))
    assert lobe[0] == 2
    f0 = 0.04 * (1 - metallic) + albedo * metallic
    fs = f0 + (1 - f0) * (1 - 0.5) ** 5
    p_spec = min(max(float(fs @ [0.2126, 0.7152, 0.0722]), 0.04), 0.9)
    lum = float(albedo @ [0.2126, 0.7152, 0.0722])
    sc = (1 - tint) + albedo / lum * tint
    want = (albedo * (1 - metallic) + sc * sheen * (1 - metallic) * 0.5 ** 5 * math.pi) / (1 - p_spec)
    np.testing.assert_allclose(att[0], want, rtol=1e-5)


def test_back_facing_view_scatters_nothing():
    m = Material.pbr((0.8, 0.8, 0.8))
    lobe, _, _, _, _ = O.pbr_scatter(m, np.array([[0.0, -1.0, 0.0]]), (0.0, 1.0, 0.0), np.array([[0.5] * 4]))
    assert lobe[0] == 0


def test_pbr_toml_defaults():
    """scene_file.rs:380-406, 457-466: roughness 0.5, clearcoat_roughness 0.03,
    film_ior 1.5, sheen_tint 0.5, the rest 0."""
    doc = {"camera": {"look_from": [0, 0, -5], "look_at": [0, 0, 0]},
           "objects": [{"shape": {"type": "sphere", "center": [0, 0, 0], "radius": 1.0},
                        "material": {"type": "pbr", "albedo": [1.0, 0.78, 0.34], "metallic": 1.0}}]}
    m = scene_from_toml_dict(doc).materials[0]
    assert (m.roughness, m.metallic, m.clearcoat, m.clearcoat_roughness, m.film_ior, m.sheen_tint) == \
        pytest.approx((0.5, 1.0, 0.0, 0.03, 1.5, 0.5))
    assert m.emission_strength == 0.0 and m.anisotropy == 0.0
