"""Cylinders, cones, disks and infinite planes in the CPU oracle, pinned to the
reference's own tests (cylinder.rs:19-125, cone.rs:148-254, disk.rs:19-100)
and to the SRT placement of objects (scene_file.rs:1036-1042)."""
import math

import numpy as np
import pytest

from oracle import oracle as O
from rustracer_b200.scene import Material, SceneBuilder, Transform, scene_from_toml_dict
from tests.helpers import ray, rays


def _scene(kind, xf=None, **kw):
    sb = SceneBuilder()
    m = sb.add_material(Material.lambertian((0.5, 0.5, 0.5)))
    sb.add_shape(kind, m, xf=xf, **kw)
    return sb


def _hit(sb, o, d, tmin=0.001, tmax=np.inf):
    rs = rays(ray(o, d, tmin, tmax))
    h = O.OracleScene(sb).trace_closest(rs)[0]
    return None if h["prim"] < 0 else h


def _part(h):
    return int(np.array([h["b1"]], np.float32).view(np.int32)[0])


CYL = dict(center=(0, 0, 0), radius=1.0, height=2.0)
CONE = dict(center=(0, 0, 0), radius=1.0, height=2.0)


def test_cylinder_known_answers():
    sb = _scene("cylinder", **CYL)
    h = _hit(sb, (0, 1, -5), (0, 0, 1))
    assert abs(h["t"] - 4.0) < 1e-5 and _part(h) == 0                # lateral, t = 4
    h = _hit(sb, (0, -5, 0), (0, 1, 0))
    assert abs(h["t"] - 5.0) < 1e-5 and _part(h) == 1                # bottom cap
    h = _hit(sb, (0, 5, 0), (0, -1, 0))
    assert abs(h["t"] - 3.0) < 1e-5 and _part(h) == 2                # top cap
    assert _hit(sb, (2, 1, -5), (0, 0, 1)) is None                   # outside the radius
    assert _hit(sb, (0, 3, -5), (0, 0, 1)) is None                   # above the height
    # the closed endpoint t == t_max is a hit (cylinder.rs:97-114)
    assert abs(_hit(sb, (0, 1, -5), (0, 0, 1), tmax=4.0)["t"] - 4.0) < 1e-6
    assert _hit(sb, (0, 1, -5), (0, 0, 1), tmax=np.float32(4.0) - np.float32(1e-4)) is None


def test_cone_known_answers():
    sb = _scene("cone", **CONE)
    h = _hit(sb, (0, 1, -5), (0, 0, 1))
    assert abs(h["t"] - 4.5) < 1e-5 and _part(h) == 0                # lateral: radius 0.5 at y = 1
    h = _hit(sb, (0.5, -5, 0), (0, 1, 0))
    assert abs(h["t"] - 5.0) < 1e-5 and _part(h) == 1                # base cap
    assert _hit(sb, (2, 1, -5), (0, 0, 1)) is None
    assert _hit(sb, (0, 3, -5), (0, 0, 1)) is None
    assert abs(_hit(sb, (0, 1, -5), (0, 0, 1), tmax=4.5)["t"] - 4.5) < 1e-5
    assert _hit(sb, (0, 1, -5), (0, 0, 1), tmax=np.float32(4.5) - np.float32(1e-4)) is None
    assert abs(_hit(sb, (0.5, -5, 0), (0, 1, 0), tmax=5.0)["t"] - 5.0) < 1e-5


def test_disk_known_answers():
    sb = _scene("disk", center=(0, 0, 0), normal=(0, 0, 1), radius=1.0)
    assert abs(_hit(sb, (0, 0, 2), (0, 0, -1))["t"] - 2.0) < 1e-5
    assert _hit(sb, (0.99, 0, 1), (0, 0, -1)) is not None
    assert _hit(sb, (1.01, 0, 1), (0, 0, -1)) is None
    assert _hit(sb, (0, 0, 0), (1, 0, 0)) is None                     # parallel
    assert _hit(sb, (0, 0, -2), (0, 0, 1)) is not None               # back side


@pytest.mark.parametrize("kind,kw", [("cylinder", CYL), ("cone", CONE),
                                     ("disk", dict(center=(0, 0, 0), normal=(0, 0, 1), radius=1.0)),
                                     ("infinite_plane", dict(center=(0, 0, 0), normal=(0, 1, 0)))])
def test_any_hit_agrees_with_hit(kind, kw):
    sb = _scene(kind, **kw)
    rng = np.random.default_rng(2)
    o = rng.normal(0, 3, (3000, 3))
    d = rng.normal(0, 1, (3000, 3))
    rs = np.concatenate([o, d, np.full((3000, 1), 0.001), np.full((3000, 1), np.inf)], 1).astype(np.float32)
    s = O.OracleScene(sb)
    h, occ = s.trace_closest(rs), s.trace_any(rs)
    assert ((h["prim"] >= 0) == (occ != 0)).all()
    assert np.array_equal(h, s.trace_closest(rs, brute=True))


def test_infinite_plane_hits_everywhere_inside_its_proxy_box():
    sb = _scene("infinite_plane", center=(0, -1, 0), normal=(0, 1, 0), wave_amplitude=0.05, wave_scale=3.0)
    h = _hit(sb, (1234.5, 10, -987.0), (0.1, -1, 0.2))
    assert h is not None and abs(h["t"] * 1.0 - 11.0) < 1e-3        # y: 10 → −1 at unit vertical speed
    assert _hit(sb, (2e5, 10, 0), (0, -1, 0)) is None                 # beyond the ±1e5 proxy box


def test_srt_placement_matches_the_object_space_ray():
    """A scaled, rotated and translated cylinder: the oracle's hits equal those
    of the unplaced cylinder traced with the ray moved into object space by
    Translate⁻¹, Rotate⁻¹, UniformScale⁻¹ (transform.rs)."""
    xf = Transform(scale=1.5, rotate=(30.0, -20.0, 10.0), translate=(0.5, 0.2, -0.3))
    placed, plain = _scene("cylinder", xf=xf, **CYL), _scene("cylinder", **CYL)
    rng = np.random.default_rng(4)
    n = 4000
    o = rng.normal(0, 4, (n, 3))
    d = xf.point(rng.normal(0, 0.6, (n, 3)) + np.array([0, 1.0, 0])) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rw = np.concatenate([o, d, np.full((n, 1), 0.001), np.full((n, 1), np.inf)], 1).astype(np.float32)
    oo = ((o - xf.t) @ xf.R) / xf.scale
    do = (d @ xf.R) / xf.scale
    ro = np.concatenate([oo, do, np.full((n, 1), 0.001), np.full((n, 1), np.inf)], 1).astype(np.float32)
    hw = O.OracleScene(placed).trace_closest(rw)
    ho = O.OracleScene(plain).trace_closest(ro)
    both = (hw["prim"] >= 0) & (ho["prim"] >= 0)
    assert both.sum() > n // 4 and ((hw["prim"] >= 0) == (ho["prim"] >= 0)).mean() > 0.998
    np.testing.assert_allclose(hw["t"][both], ho["t"][both], rtol=1e-4, atol=1e-5)


def test_toml_shapes_and_validation():
    doc = {"camera": {"look_from": [0, 0, -5], "look_at": [0, 0, 0]},
           "objects": [{"shape": {"type": "cylinder", "center": [0, 0, 0], "radius": 0.5, "height": 1.0},
                        "material": {"type": "lambertian", "color": [0.5, 0.5, 0.5]}, "rotate": [90, 0, 0]},
                       {"shape": {"type": "cone", "center": [2, 0, 0], "radius": 0.5, "height": 1.0},
                        "material": {"type": "lambertian", "color": [0.5, 0.5, 0.5]}},
                       {"shape": {"type": "disk", "center": [0, 0, 0], "normal": [0, 1, 0], "radius": 30},
                        "material": {"type": "pbr", "albedo": [0.5, 0.48, 0.46], "roughness": 0.25}},
                       {"shape": {"type": "infinite_plane", "point": [0, -1, 0], "normal": [0, 1, 0],
                                  "wave_amplitude": 0.05}, "material": {"type": "lambertian", "color": [0.2, 0.3, 0.4]}}]}
    sb = scene_from_toml_dict(doc)
    assert [s.type for s in sb.shapes] == [0, 1, 2, 3]
    assert sb.shapes[3].wave_scale == 1.0
    O.OracleScene(sb)
    doc["objects"][2]["shape"]["normal"] = [0, 0, 0]
    with pytest.raises(ValueError, match="normal"):
        scene_from_toml_dict(doc)
