"""Analytic convex gems in the CPU oracle: the round/oval brilliant's
half-spaces (Diamond::new, diamond.rs:93-195), the convex slab test
(diamond.rs:202-253), the gem placement (transform.rs) and the [[gems]]
grading-report loader (scene_file.rs:676-931), each pinned to the reference's
own unit tests (diamond.rs:290-520, scene_file.rs:1271-1545, transform.rs:393-411)."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.scene import (Material, SceneBuilder, diamond_planes, gem_absorption, gem_geometry, gem_preset,
                                  scene_from_toml_dict)
from tests.helpers import ray, rays

PI = math.pi


def _diamond(**kw):
    sb = SceneBuilder()
    m = sb.add_material(Material.dielectric(1.5))
    sb.add_diamond((0.0, 0.0, 0.0), 1.0, m, **kw)
    return sb


def _hits(sb, rs):
    s = O.OracleScene(sb)
    h = s.trace_closest(rs)
    return s, h


def _plane_idx(h):
    return h["b1"].view(np.int32)


def _normals(sb, h, rs):
    """Face-forward geometric normals of unpolished hits (hittable.rs:89-93)."""
    c = sb.convex[0]
    R = c["rot"]
    n = c["planes"][_plane_idx(h), :3].astype(np.float64) @ R.T
    front = (rs[:, 3:6] * n).sum(1) < 0
    return np.where(front[:, None], n, -n)


# ── plane counts (diamond.rs:379-392, 501-507, 436-438) ───────────────────────
def test_plane_counts():
    assert len(diamond_planes((0, 0, 0), 1.0, girdle_facets=64)[0]) == 193
    assert len(diamond_planes((0, 0, 0), 1.0)[0]) == 97
    assert len(diamond_planes((0, 0, 0), 1.0, girdle_facets=17)[0]) == 97
    assert len(diamond_planes((0, 0, 0), 1.0, girdle_pct=0.0)[0]) == 17
    assert len(diamond_planes((0, 0, 0), 1.0, girdle_finish="faceted")[0]) == 49


# ── pavilion facets (diamond.rs:290-315) ──────────────────────────────────────
def test_pavilion_has_n_facets_converging_at_culet():
    sb = _diamond(girdle_facets=16, girdle_pct=2.0)
    pav_h = math.tan(math.radians(40.75))
    y = -pav_h * 0.5
    rs = rays(*[ray((0, y, 0), (math.cos(i * PI / 360), 0, math.sin(i * PI / 360))) for i in range(720)])
    _, h = _hits(sb, rs)
    assert (h["prim"] >= 0).all()
    nrm = _normals(sb, h, rs)
    P = sb.convex[0]["planes"][:, :3]
    seen = set()
    for v in nrm:
        for k, pn in enumerate(P):
            if np.linalg.norm(v - pn) < 1e-4 or np.linalg.norm(v + pn) < 1e-4:
                seen.add(k)
                break
    assert len(seen) == 16


# ── girdle outlines (diamond.rs:317-364) ──────────────────────────────────────
@pytest.mark.parametrize("finish,n,m", [("faceted", 720, 16), ("uniform", 1440, 64), ("polished", 1440, 64)])
def test_girdle_outline(finish, n, m):
    sb = _diamond(girdle_facets=16, girdle_pct=2.0, girdle_finish=finish)
    rs = rays(*[ray((0, 0, 0), (math.cos(i * 2 * PI / n), 0, math.sin(i * 2 * PI / n))) for i in range(n)])
    _, h = _hits(sb, rs)
    assert (h["prim"] >= 0).all()
    dist = h["t"]                                  # unit directions from the centre
    assert abs(dist.min() - 1.0) < 1e-3
    assert abs(dist.max() - 1.0 / math.cos(PI / m)) < 1e-3


# ── the closed entry interval (diamond.rs:367-376) ────────────────────────────
def test_convex_hit_accepts_entry_at_exactly_t_max():
    # the slab x ∈ [-1, 1] closed by far planes in y and z (the API wants ≥ 4 planes)
    pl = np.array([[1, 0, 0, 1], [-1, 0, 0, 1], [0, 1, 0, 50], [0, -1, 0, 50], [0, 0, 1, 50], [0, 0, -1, 50]],
                  np.float32)
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_convex(pl, m, (-1, -50, -50), (1, 50, 50))
    s = O.OracleScene(sb)
    h = s.trace_closest(rays(ray((-5, 0, 0), (1, 0, 0), 0.001, 4.0),
                             ray((-5, 0, 0), (1, 0, 0), 0.001, np.float32(4.0) - np.float32(1e-4))))
    assert h["prim"][0] == 0 and abs(h["t"][0] - 4.0) < 1e-6
    assert h["prim"][1] == -1


# ── oval girdle (diamond.rs:394-406) ──────────────────────────────────────────
@pytest.mark.parametrize("n", [16, 64])
def test_oval_girdle_extreme_x_is_q_times_radius(n):
    sb = _diamond(oval_ratio=1.4, girdle_facets=n)
    _, h = _hits(sb, rays(ray((10, 0, 0), (-1, 0, 0), 0.001, 100.0)))
    assert h["prim"][0] == 0 and abs(10.0 - h["t"][0] - 1.4) < 1e-4


# ── any-hit agrees with closest-hit (diamond.rs:408-429) ──────────────────────
def test_any_hit_agrees_with_hit():
    sb = _diamond(oval_ratio=1.4, girdle_facets=64)
    rs = rays(*[ray(o, d, 0.001, 100.0) for o, d in [
        ((0, 10, 0), (0, -1, 0)), ((10, 0, 0), (-1, 0, 0)), ((10, 0, 10), (-1, 0, -1)),
        ((0, 0.3, 0), (1, 0, 0)), ((0, 10, 3), (0, -1, 0)), ((0, -10, 0), (0, 1, 0))]])
    s, h = _hits(sb, rs)
    occ = s.trace_any(rs)
    assert ((h["prim"] >= 0) == (occ != 0)).all()
    assert (h["prim"] >= 0).tolist() == [True, True, True, True, False, True]


# ── girdle band (diamond.rs:431-500) ──────────────────────────────────────────
def _edge_rays(y):
    return rays(*[ray((10 * math.cos(k * 2 * PI / 16), y, 10 * math.sin(k * 2 * PI / 16)),
                      (-math.cos(k * 2 * PI / 16), 0, -math.sin(k * 2 * PI / 16)), 0.001, 100.0) for k in range(16)])


def test_faceted_girdle_alternates_band_facets():
    sb = _diamond(girdle_finish="faceted")
    rs = _edge_rays(0.019)
    _, h = _hits(sb, rs)
    n = _normals(sb, h, rs)
    for k in range(16):
        if k % 2 == 0:
            assert abs(n[k, 1]) < 1e-6
        else:
            assert n[k, 1] > 0.5


def test_uniform_girdle_keeps_band_at_every_vertex():
    sb = _diamond()
    rs = _edge_rays(0.019)
    _, h = _hits(sb, rs)
    assert (np.abs(_normals(sb, h, rs)[:, 1]) < 1e-6).all()


def test_girdle_band_is_a_flat_vertical_ring():
    sb = _diamond()
    rs = rays(ray((10, 0, 0), (-1, 0, 0), 0.001, 100.0))
    _, h = _hits(sb, rs)
    assert abs(10.0 - h["t"][0] - 1.0) < 1e-4
    assert abs(_normals(sb, h, rs)[0, 1]) < 1e-6
    lo, hi = sb.convex[0]["lo"], sb.convex[0]["hi"]
    crown_h = (1.0 - 0.53) * math.tan(math.radians(34.5))
    assert abs(hi[1] - (0.02 + crown_h)) < 1e-4
    assert abs(lo[1] + (0.02 + math.tan(math.radians(40.75)))) < 1e-4


def test_band_height_is_uniform_on_every_edge():
    sb = _diamond()
    for y, sign in ((0.021, 1), (-0.021, -1)):
        rs = _edge_rays(y)
        _, h = _hits(sb, rs)
        assert (sign * _normals(sb, h, rs)[:, 1] > 0.5).all()


def test_round_default_still_hits_table_from_above():
    sb = _diamond()
    rs = rays(ray((0, 10, 0), (0, -1, 0), 0.001, 100.0))
    _, h = _hits(sb, rs)
    py = 10.0 - h["t"][0]
    assert 0.0 < py < 10.0
    assert abs(_normals(sb, h, rs)[0, 1] - 1.0) < 1e-5


# ── placement (transform.rs:393-411; scene_file.rs:924-930) ───────────────────
def test_rotation_about_the_gem_center_keeps_it_in_place():
    """Rotate::euler_about turns the stone in place: a 180° spin about y of a
    gem at (2,0,0) leaves its table where it was, and an x-tilt of 90° about
    its own centre turns the table normal to +z."""
    for ang, d, n_exp in (((0, 180, 0), (0, -1, 0), (0, 1, 0)), ((90, 0, 0), (0, 0, -1), (0, 0, 1))):
        sb = SceneBuilder()
        m = sb.add_material(Material.dielectric(1.5))
        sb.add_diamond((2.0, 0.0, 0.0), 1.0, m, rotate=ang)
        o = np.array([2.0, 0.0, 0.0]) - 10 * np.array(d, float)
        rs = rays(ray(o, d, 0.001, 100.0))
        _, h = _hits(sb, rs)
        assert h["prim"][0] == 0
        n = _normals(sb, h, rs)[0]
        assert np.allclose(n, n_exp, atol=1e-5), n


def test_placement_matches_the_object_space_ray_transform():
    """World-space planes give the same hits as the reference's route: the
    ray moved into object space by Translate⁻¹, Rotate⁻¹ about the pivot and
    UniformScale⁻¹ (transform.rs:29-45, 228-242), then the unplaced solid."""
    rng = np.random.default_rng(5)
    s, R_deg, t, c = 1.7, (20.0, -35.0, 50.0), np.array([0.3, -0.2, 0.5]), np.array([0.5, 0.25, -0.4])
    placed, plain = SceneBuilder(), SceneBuilder()
    m1, m2 = placed.add_material(Material.dielectric(1.5)), plain.add_material(Material.dielectric(1.5))
    placed.add_diamond(c, 0.6, m1, scale=s, rotate=R_deg, translate=t)
    plain.add_diamond(c, 0.6, m2)
    R = placed.convex[0]["rot"]
    n = 4000
    target = (R @ (s * c - c) + c + t) + rng.normal(0, 0.4, (n, 3))
    o = rng.normal(0, 1, (n, 3))
    o = 4.0 * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rw = np.concatenate([o, d, np.full((n, 1), 0.001), np.full((n, 1), np.inf)], 1).astype(np.float32)
    # object space: x = (Rᵀ(x_w − c − t) + c) / s; t is invariant under the uniform scale
    oo = ((o - c - t) @ R + c) / s
    do = (d @ R) / s
    ro = np.concatenate([oo, do, np.full((n, 1), 0.001), np.full((n, 1), np.inf)], 1).astype(np.float32)
    _, hw = _hits(placed, rw)
    _, ho = _hits(plain, ro)
    hit_w, hit_o = hw["prim"] >= 0, ho["prim"] >= 0
    assert hit_w.sum() > n // 4
    agree = hit_w == hit_o
    assert agree.mean() > 0.998                    # grazing rays may flip by one rounding
    both = hit_w & hit_o
    assert np.allclose(hw["t"][both], ho["t"][both], rtol=1e-4, atol=1e-5)
    same_face = _plane_idx(hw)[both] == _plane_idx(ho)[both]
    assert same_face.mean() > 0.995


# ── [[gems]] loader (scene_file.rs:1271-1545) ─────────────────────────────────
def _gem_doc(**g):
    g.setdefault("center", [0, 0, 0])
    return {"name": "t", "camera": {"look_from": [0, 0, -1], "look_at": [0, 0, 0]},
            "background": {"type": "solid", "color": [0, 0, 0]}, "gems": [g]}


def _gem_box(**g):
    sb = scene_from_toml_dict(_gem_doc(**g))
    c = sb.convex[0]
    return np.array(c["lo"]), np.array(c["hi"])


def test_gem_carat_maps_to_girdle_diameter():
    lo, hi = _gem_box(carat=1.0)
    expected = np.float32(np.cbrt(np.float32(1.0) / np.float32(0.00355))) * 0.001 / math.cos(PI / 64)
    assert abs((hi[0] - lo[0]) - expected) < 1e-6


def test_gem_measurements_override_carat():
    lo, hi = _gem_box(carat=99.0, measurements_mm=[6.50, 6.40, 4.01])
    assert abs((hi[0] - lo[0]) - 6.40 * 0.001 / math.cos(PI / 64)) < 1e-6


def test_gem_requires_a_size_source():
    with pytest.raises(ValueError, match="carat or measurements_mm"):
        scene_from_toml_dict(_gem_doc())


def test_gem_oval_measurements_set_ratio_and_radius():
    lo, hi = _gem_box(measurements_mm=[8.99, 6.42, 3.97], table_pct=58.0)
    wx, wz = hi[0] - lo[0], hi[2] - lo[2]
    assert abs(wz - 6.42 * 0.001 / math.cos(PI / 64)) < 1e-6
    assert abs(wx / wz - 8.99 / 6.42) < 1e-4
    assert len(scene_from_toml_dict(_gem_doc(measurements_mm=[8.99, 6.42, 3.97])).convex[0]["planes"]) == 193


def test_gem_igi_percentages_convert_to_angles():
    g = dict(measurements_mm=[8.99, 6.42, 3.97], table_pct=58.0, crown_pct=16.0, pavilion_pct=41.0)
    lo, hi = _gem_box(**g)
    h_mm = (hi[1] - lo[1]) / 0.001
    assert abs(h_mm - (0.02 + 0.16 + 0.41) * 6.42) < 0.02
    geo = gem_geometry(g)
    assert abs(geo["crown_angle"] - 37.3) < 0.2 and abs(geo["pavilion_angle"] - 39.35) < 0.2


def test_gem_defaults_to_tolkowsky_cut():
    geo = gem_geometry(dict(carat=0.5, center=[0, 0, 0]))
    assert (geo["table_pct"], geo["crown_angle"], geo["pavilion_angle"]) == (53.0, 34.5, 40.75)
    assert geo["girdle_facets"] == 16 and geo["girdle_finish"] == "uniform"


def test_gem_material_presets():
    d, s, r, e = (gem_preset(k) for k in ("diamond", "sapphire", "ruby", "emerald"))
    assert abs(d[0] - 2.351) < 1e-6 and not any(d[2])
    # Cauchy n(λ) = B + C/λ²  (λ in µm): diamond's nF − nC ≈ 0.044
    n = lambda b, c, lam: b + c / (lam / 1000.0) ** 2
    assert abs(n(d[0], d[1], 486.1) - n(d[0], d[1], 656.3) - 0.044) < 0.002
    assert abs(s[0] - 1.741) < 1e-6 and abs(e[0] - 1.556) < 1e-6
    assert s[2][0] > 100 and s[2][2] < 100
    assert r[2][1] > 100 and r[2][0] < 100
    assert e[2][1] < 100 and e[2][0] > 100 and e[2][2] > 100
    with pytest.raises(ValueError):
        gem_preset("topaz")


def test_gem_absorption_rescales_with_scale_mm():
    ruby = gem_preset("ruby")[2]
    base = dict(measurements_mm=[5.0, 5.0, 3.0], material="ruby", color_grade="F", center=[0, 0, 0])
    a_m = gem_absorption(dict(base, scale_mm=0.001), ruby)
    assert abs(a_m[0] - 25.0) < 1e-4 and abs(a_m[1] - 550.0) < 1e-3
    a_n = gem_absorption(dict(base, scale_mm=0.2), ruby)
    assert abs(a_n[0] - 25.0 * 0.005) < 1e-5 and abs(a_n[1] - 550.0 * 0.005) < 1e-4
    a_x = gem_absorption(dict(base, scale_mm=0.2, absorption=[1.0, 2.0, 3.0]), ruby)
    assert abs(a_x[2] - (450.0 * 0.005 + 3.0)) < 1e-4
    a_k = gem_absorption(dict(carat=1.0, color_grade="K", center=[0, 0, 0], scale_mm=0.001), (0.0, 0.0, 0.0))
    assert abs(a_k[0] - 230.0) < 1e-3


def test_gem_girdle_finish_parses_and_validates():
    sb = scene_from_toml_dict(_gem_doc(measurements_mm=[5.0, 5.0, 3.0], girdle_finish="faceted"))
    assert len(sb.convex[0]["planes"]) == 49
    with pytest.raises(ValueError, match="girdle_finish"):
        scene_from_toml_dict(_gem_doc(measurements_mm=[5.0, 5.0, 3.0], girdle_finish="rough"))


def test_gem_unknown_cut_or_material_errors():
    with pytest.raises(ValueError, match="material"):
        scene_from_toml_dict(_gem_doc(carat=1.0, material="topaz"))
    with pytest.raises(ValueError, match="cut"):
        scene_from_toml_dict(_gem_doc(carat=1.0, cut="heart"))


def test_gem_spin_and_rotate_pivot_on_the_center():
    sb = scene_from_toml_dict(_gem_doc(measurements_mm=[5.0, 5.0, 3.0], center=[0.0, 0.5, 0.0], rotate=[10.0, 0.0, 0.0],
                                       spin=30.0))
    c = sb.convex[0]
    assert c["pivot"] == (0.0, 0.5, 0.0)
    R = c["rot"]
    assert np.allclose(R @ R.T, np.eye(3), atol=1e-12) and not np.allclose(R, np.eye(3))
    s = O.OracleScene(sb)
    h = s.trace_closest(rays(ray((0, 0.5, -1), (0, 0, 1))))
    assert h["prim"][0] == 0                       # still centred at (0, 0.5, 0)


def test_invalid_cut_parameters_error():
    with pytest.raises(ValueError, match="table_pct"):
        scene_from_toml_dict(_gem_doc(carat=1.0, table_pct=120.0))
    with pytest.raises(ValueError, match="pavilion angle"):
        scene_from_toml_dict({"camera": {"look_from": [0, 0, -1], "look_at": [0, 0, 0]},
                              "objects": [{"shape": {"type": "diamond", "center": [0, 0, 0], "radius": 1.0,
                                                     "pavilion_angle": float("nan")},
                                           "material": {"type": "dielectric", "ior": 1.5}}]})


def test_polish_tilts_the_shading_normal_only():
    """A polished gem (polish > 0) keeps the same hits; only the shading normal
    moves (diamond.rs:266-270).  The hits must equal the unpolished solid's."""
    a, b = _diamond(polish=0.0), _diamond(polish=0.05)
    rng = np.random.default_rng(9)
    o = rng.normal(0, 1, (2000, 3))
    o = 3.0 * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = rng.normal(0, 0.3, (2000, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rs = np.concatenate([o, d, np.full((2000, 1), 0.001), np.full((2000, 1), np.inf)], 1).astype(np.float32)
    _, ha = _hits(a, rs)
    _, hb = _hits(b, rs)
    assert np.array_equal(ha, hb)


def test_interior_rays_in_overlapping_gems_are_order_independent():
    """A ray inside two overlapping stones crosses the nearer exit.  The
    reference's slab test also reports a phantom crossing at t_max for a solid
    whose exit lies beyond it; here a solid with no crossing in [tmin, tmax]
    is no hit, so the BVH and the brute-force scan agree on every ray."""
    sb = SceneBuilder()
    m = sb.add_material(Material.dielectric(1.5))
    sb.add_diamond((-0.3, 0.0, 0.0), 1.0, m)
    sb.add_diamond((0.3, 0.0, 0.0), 1.0, m, rotate=(0.0, 20.0, 0.0))
    rng = np.random.default_rng(4)
    o = np.stack([rng.uniform(-0.4, 0.4, 8000), rng.uniform(-0.3, 0.2, 8000), rng.uniform(-0.4, 0.4, 8000)], 1)
    for c in sb.convex:                            # keep origins strictly inside both stones
        P = c["planes"].astype(np.float64)
        nw = P[:, :3] @ c["rot"].T
        dw = (nw * (np.array(c["pivot"]) + np.array(c["translate"]))).sum(1) + c["scale"] * P[:, 3] - \
            (P[:, :3] * np.array(c["pivot"])).sum(1)
        o = o[((o @ nw.T) < dw[None, :] - 1e-3).all(1)]
    n = len(o)
    assert n > 2000
    d = rng.normal(0, 1, (n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rs = np.concatenate([o, d, np.full((n, 1), 0.001), np.full((n, 1), np.inf)], 1).astype(np.float32)
    s = O.OracleScene(sb)
    h, hb = s.trace_closest(rs), s.trace_closest(rs, brute=True)
    assert (h["prim"] >= 0).all() and np.array_equal(h, hb)
    assert (_plane_idx(h) >= 0).all()
    # the nearer of the two exits, from the planes directly (float64)
    t_exit = []
    for c in sb.convex:
        P = c["planes"].astype(np.float64) @ np.eye(4)
        R = c["rot"]
        nw = P[:, :3] @ R.T
        dw = (nw * (np.array(c["pivot"]) + np.array(c["translate"]))).sum(1) + c["scale"] * P[:, 3] - \
            (P[:, :3] * np.array(c["pivot"])).sum(1)
        nd = d @ nw.T
        tf = (dw[None, :] - o @ nw.T) / nd
        t_exit.append(np.where(nd > 0, tf, np.inf).min(1))
    np.testing.assert_allclose(h["t"], np.minimum(*t_exit), rtol=1e-4, atol=1e-5)
