"""Step-family gem cuts in the CPU oracle: StepCut::new's half-spaces
(step_cut.rs:232-392) traced through the convex primitive, pinned to the
reference's own tests (step_cut.rs:420-670) and to the [[gems]] step-cut
tests (scene_file.rs:1470-1545)."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.scene import Material, SceneBuilder, scene_from_toml_dict, step_cut_planes
from tests.helpers import ray, rays

# the reference tests' base parameters: table 50 %, 45° / 45°, chamfer 20 %,
# 3 + 3 steps, culet 8 %, spread 0.25, no girdle band
BASE = dict(table_pct=50.0, crown_angle=45.0, pavilion_angle=45.0, outline=("rect", 20.0))


def _cut(a=2.0, b=1.0, **kw):
    p = dict(BASE)
    p.update(kw)
    sb = SceneBuilder()
    m = sb.add_material(Material.dielectric(1.5))
    sb.add_step_cut((0.0, 0.0, 0.0), a, b, m, **p)
    return sb


def _hit(sb, o, d):
    rs = rays(ray(o, np.asarray(d, float) / np.linalg.norm(d), 0.001, 100.0))
    h = O.OracleScene(sb).trace_closest(rs)[0]
    if h["prim"] < 0:
        return None
    pl = sb.convex[0]["planes"][np.array([h["b1"]], np.float32).view(np.int32)[0]]
    n = pl[:3].astype(np.float64)
    front = float(np.dot(rs[0, 3:6], n)) < 0
    p = rs[0, :3].astype(np.float64) + float(h["t"]) * rs[0, 3:6].astype(np.float64)
    return p, (n if front else -n), front


def _planes(a=2.0, b=1.0, **kw):
    p = dict(BASE)
    p.update(kw)
    return step_cut_planes((0, 0, 0), a, b, **p)


def test_plane_count_is_caps_plus_edges_times_steps_plus_vertex_chevrons():
    assert len(_planes()[0]) == 2 + 8 * (3 + 3)
    assert len(_planes(crown_steps=1, pavilion_steps=2)[0]) == 2 + 8 * (1 + 2)
    assert len(_planes(outline=("triangle",), chevrons=2)[0]) == 2 + 3 * (3 + 3) + 2 * 3 * 2


def test_bbox_matches_outline_and_heights():
    _, lo, hi = _planes()
    assert abs(lo[0] + 2) < 1e-6 and abs(hi[0] - 2) < 1e-6
    assert abs(lo[2] + 1) < 1e-6 and abs(hi[2] - 1) < 1e-6
    assert abs(hi[1] - 0.5) < 1e-6 and abs(lo[1] + 0.92) < 1e-6


def test_girdle_band_adds_vertical_faces_and_height():
    pl, lo, hi = _planes(girdle_pct=10.0)
    assert len(pl) == 2 + 8 + 8 * (3 + 3)
    p, n, _ = _hit(_cut(girdle_pct=10.0), (10, 0, 0), (-1, 0, 0))
    assert abs(p[0] - 2.0) < 1e-4 and abs(n[1]) < 1e-6
    assert abs(hi[1] - 0.6) < 1e-4 and abs(lo[1] + 1.02) < 1e-4


def test_horizontal_ray_hits_girdle_edge_at_semi_axis():
    p, _, _ = _hit(_cut(), (10, 0, 0), (-1, 0, 0))
    assert abs(p[0] - 2.0) < 1e-4 and abs(p[1]) < 1e-4


def test_diagonal_ray_hits_chamfer_not_the_sharp_corner():
    sb = _cut()
    target = np.array([1.9, 0.0, 0.9])
    p, _, _ = _hit(sb, (10, 0, 5), target - np.array([10, 0, 5]))
    assert abs(p[0] + p[2] - 2.8) < 1e-4 and p[0] + p[2] < 2.9
    p2, _, _ = _hit(sb, (10, 0, 10), (-1, 0, -1))
    assert abs(p2[2] - 1.0) < 1e-4


def test_zero_corner_pct_gives_sharp_square_corners():
    assert len(_planes(1.0, 1.0, outline=("rect", 0.0))[0]) == 2 + 4 * (3 + 3)
    p, _, _ = _hit(_cut(1.0, 1.0, outline=("rect", 0.0)), (10, 0, 10), (-1, 0, -1))
    assert abs(p[0] + p[2] - 2.0) < 1e-4


def test_ray_from_above_hits_table_with_up_normal():
    p, n, _ = _hit(_cut(), (0, 10, 0), (0, -1, 0))
    assert abs(p[1] - 0.5) < 1e-5 and abs(n[1] - 1.0) < 1e-5


def test_interior_ray_exits_through_side():
    p, n, front = _hit(_cut(), (0, 0.25, 0), (1, 0, 0))
    assert p[0] > 1.0 and not front and n[0] < 0


def test_chevron_planes_keep_outline_and_bbox():
    kw = dict(outline=("rect", 0.0), chevrons=2)
    pl, lo, hi = _planes(1.0, 1.0, **kw)
    assert len(pl) == 2 + 4 * (3 + 3) + 8 * 2
    p, _, _ = _hit(_cut(1.0, 1.0, **kw), (10, 0, 10), (-1, 0, -1))
    assert abs(p[0] + p[2] - 2.0) < 1e-4
    assert abs(hi[0] - 1.0) < 1e-6 and abs(hi[2] - 1.0) < 1e-6


def test_chevron_plane_cuts_crown_near_corner():
    p, n, _ = _hit(_cut(1.0, 1.0, outline=("rect", 0.0), chevrons=2), (0.9, 10, 0.9), (0, -1, 0))
    assert p[1] < 0.5 - 1e-3
    assert abs(n[0] - n[2]) < 1e-4 and n[0] > 0.1


def test_triangle_outline_is_pointed_and_bounded():
    sb = _cut(outline=("triangle",))
    p, _, _ = _hit(sb, (0, 0, 10), (0, 0, -1))
    assert abs(p[2] - 1.0) < 1e-4
    p, _, _ = _hit(sb, (10, 0, 0), (-1, 0, 0))
    assert abs(p[0] - 2.0 / math.sqrt(3.0)) < 1e-4


def test_marquise_outline_has_pointed_tips():
    kw = dict(outline=("pointed_oval", 16, False))
    p, _, _ = _hit(_cut(2.0, 0.5, **kw), (10, 0, 0), (-1, 0, 0))
    assert abs(p[0] - 2.0) < 1e-3
    _, lo, hi = _planes(2.0, 0.5, **kw)
    assert abs(hi[0] - 2.0) < 1e-6 and abs(hi[2] - 0.5) < 1e-6


def test_rounded_rect_arc_reaches_full_extents():
    _, lo, hi = _planes(outline=("rounded_rect", 30.0, 4))
    assert abs(hi[0] - 2.0) < 1e-6 and abs(lo[0] + 2.0) < 1e-6
    assert abs(hi[2] - 1.0) < 1e-6 and abs(lo[2] + 1.0) < 1e-6


def test_table_pct_is_exact_under_step_spread():
    sb = SceneBuilder()
    sb.add_step_cut((0, 0, 0), 1.0, 1.0, sb.add_material(Material.dielectric(1.5)), table_pct=50.0,
                    crown_angle=45.0, pavilion_angle=45.0, outline=("rect", 0.0))
    inside, _, _ = _hit(sb, (0.49, 10, 0), (0, -1, 0))
    outside, _, _ = _hit(sb, (0.51, 10, 0), (0, -1, 0))
    assert abs(inside[1] - 0.5) < 1e-4 and outside[1] < 0.5 - 1e-3


def test_polygon_outline_validation():
    with pytest.raises(ValueError, match="convex"):
        _planes(1.0, 1.0, outline=("polygon", [[1, 0], [0, 1], [0.2, 0.2], [-1, 0], [0, -1]]))
    _planes(1.0, 1.0, outline=("polygon", [[0, 1], [0, 1], [-0.866, -0.5], [0.866, -0.5]]))
    with pytest.raises(ValueError, match="3 distinct"):
        _planes(1.0, 1.0, outline=("polygon", [[1, 0], [1, 0]]))


def test_invalid_params_error_not_panic():
    for kw in (dict(crown_angle=0.0), dict(crown_angle=95.0)):
        with pytest.raises(ValueError):
            _planes(1.0, 1.0, **kw)
    for a in (0.0, -1.0):
        with pytest.raises(ValueError):
            _planes(a, 1.0)


def test_any_hit_agrees_with_hit():
    for outline in (("rect", 0.0), ("rounded_rect", 30.0, 4)):
        sb = _cut(outline=outline, chevrons=2)
        rs = rays(*[ray(o, d, 0.001, 100.0) for o, d in [
            ((0, 10, 0), (0, -1, 0)), ((10, 0, 0), (-1, 0, 0)), ((10, 0, 10), (-1, 0, -1)),
            ((0, 0.25, 0), (1, 0, 0)), ((0, 10, 5), (0, -1, 0)), ((0, -10, 0), (0, 1, 0))]])
        s = O.OracleScene(sb)
        h, occ = s.trace_closest(rs), s.trace_any(rs)
        assert ((h["prim"] >= 0) == (occ != 0)).all()
        assert (h["prim"] >= 0).tolist() == [True, True, True, True, False, True]


def test_steps_make_visibly_different_planes():
    pl = _planes()[0]
    crown = [q for q in pl if q[1] > 0.3 and q[0] > 0.5 and abs(q[2]) < 1e-6]
    assert len(crown) >= 3 and abs(crown[0][1] - crown[2][1]) > 0.05


# ── [[gems]] step cuts (scene_file.rs:1470-1530) ──────────────────────────────
def _gem_box(**g):
    g.setdefault("center", [0, 0, 0])
    sb = scene_from_toml_dict({"camera": {"look_from": [0, 0, -1], "look_at": [0, 0, 0]}, "gems": [g]})
    c = sb.convex[0]
    return np.array(c["hi"]) - np.array(c["lo"]), sb


def test_gem_step_cut_uses_measurements_as_rectangle():
    ext, _ = _gem_box(measurements_mm=[9.0, 6.0, 3.9], cut="step", material="emerald")
    assert abs(ext[0] - 0.009) < 1e-6 and abs(ext[2] - 0.006) < 1e-6


def test_gem_princess_cut_is_square_and_takes_chevrons():
    ext, sb = _gem_box(measurements_mm=[7.0, 7.0, 4.2], cut="princess", material="sapphire")
    assert abs(ext[0] - 0.007) < 1e-6 and abs(ext[2] - 0.007) < 1e-6
    # 4 edges × (band + 4 + 4) + 4 vertices × 2 × 3 chevrons + 2 caps
    assert len(sb.convex[0]["planes"]) == 4 * 9 + 24 + 2
    ext, sb = _gem_box(measurements_mm=[7.0, 7.0, 4.2], cut="princess", chevrons=2)
    assert abs(ext[0] - 0.007) < 1e-6 and len(sb.convex[0]["planes"]) == 4 * 9 + 16 + 2


def test_gem_trillion_and_marquise_build():
    ext, _ = _gem_box(measurements_mm=[7.0, 7.0, 4.2], cut="trillion")
    a = 0.0035
    assert abs(ext[0] - 2 * 0.866 * a) < 1e-5 and abs(ext[2] - 1.5 * a) < 1e-5
    ext, sb = _gem_box(measurements_mm=[10.0, 4.0, 3.0], cut="marquise")
    assert abs(ext[0] - 0.010) < 1e-6 and abs(ext[2] - 0.004) < 1e-6
    assert len(sb.convex[0]["planes"]) == 48 * 9 + 48 * 2 * 2 + 2     # within the 1024-plane limit
    O.OracleScene(sb)


def test_step_cut_object_shape():
    doc = {"camera": {"look_from": [0, 0, -5], "look_at": [0, 0, 0]},
           "objects": [{"shape": {"type": "step_cut", "center": [0, 0, 0], "length": 4.0, "width": 2.0,
                                  "outline": "hexagon", "chevrons": 1},
                        "material": {"type": "dielectric", "ior": 1.5}}]}
    sb = scene_from_toml_dict(doc)
    assert len(sb.convex[0]["planes"]) == 2 + 6 * (1 + 3 + 3) + 6 * 2
    doc["objects"][0]["shape"]["outline"] = "polygon"
    with pytest.raises(ValueError, match="points"):
        scene_from_toml_dict(doc)
