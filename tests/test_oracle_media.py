"""Participating media in the CPU oracle, pinned to the reference's own unit
tests of volume.rs (cited per test), plus the scatter-distance law."""
import math

import numpy as np

from oracle import oracle as O
from tests.helpers import medium_sphere_scene, ray, rays


def test_constant_medium_beer_lambert():
    # volume.rs:280-307
    s = O.OracleScene(medium_sphere_scene())
    tr = s.trace_transmittance(rays(
        ray((-5, 0, 0), (1, 0, 0)),                 # chord 2 → exp(-2)
        ray((-5, 5, 0), (1, 0, 0)),                 # misses the boundary → 1
        ray((0, 0, 0), (1, 0, 0)),                  # origin inside: [0.001, 1] → exp(-0.999)
        ray((0, 0, 0), (1, 0, 0), tmax=0.5),        # t_max inside: [0.001, 0.5]
    ))
    assert abs(tr[0] - math.exp(-2.0)) < 1e-6
    assert tr[1] == 1.0
    assert abs(tr[2] - math.exp(-0.999)) < 1e-6
    assert abs(tr[3] - math.exp(-(0.5 - 0.001))) < 1e-5
    # volumes never occlude through any_hit
    assert s.trace_any(rays(ray((-5, 0, 0), (1, 0, 0))))[0] == 0


def test_transmittance_composes_across_list():
    # volume.rs:309-325
    s = O.OracleScene(medium_sphere_scene(blocker=True))
    tr = s.trace_transmittance(rays(ray((-5, 0, 0), (1, 0, 0)), ray((-5, 0.9, 0), (1, 0, 0))))
    assert tr[0] == 0.0
    l = 2.0 * math.sqrt(1.0 - 0.9 * 0.9)
    assert abs(tr[1] - math.exp(-l)) < 1e-5


def test_hg_sample_finite_at_extreme_g():
    # volume.rs:327-339
    rng = np.random.default_rng(1)
    w = np.tile(np.array([0, 0, 1], np.float32), (20000, 1))
    for g in (1.0, -1.0, 0.999999, -0.999999):
        d = O.hg_sample(w, g, rng.random(20000), rng.random(20000))
        assert np.isfinite(d).all()


def test_hg_sample_mean_cosine_is_g():
    # the HG phase function has ⟨cos θ⟩ = g (volume.rs:14-20)
    rng = np.random.default_rng(2)
    w = np.tile(np.array([0, 0, 1], np.float32), (200000, 1))
    for g in (0.0, 0.3, -0.5, 0.85):
        d = O.hg_sample(w, g, rng.random(200000), rng.random(200000))
        assert abs(d[:, 2].mean() - g) < 0.01
        assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-5)


def test_constant_medium_free_flight_is_exponential():
    # ConstantMedium::hit (volume.rs:97-138): distance −ln(ξ)/σ inside the boundary
    s = O.OracleScene(medium_sphere_scene(density=0.7))
    rng = np.random.default_rng(3)
    n = 40000
    o = np.column_stack([np.full(n, -5.0), rng.uniform(-0.05, 0.05, n), rng.uniform(-0.05, 0.05, n)])
    r = np.concatenate([o, np.tile([1.0, 0, 0], (n, 1)), np.full((n, 1), 0.001), np.full((n, 1), np.inf)], 1)
    h = s.trace_closest(r.astype(np.float32))
    hit = h["prim"] == 0                              # the medium's id follows the (zero) primitives
    entry = 5.0 - np.sqrt(1.0 - o[:, 1] ** 2 - o[:, 2] ** 2)
    chord = 2.0 * np.sqrt(1.0 - o[:, 1] ** 2 - o[:, 2] ** 2)
    p_scatter = 1.0 - np.exp(-0.7 * chord)
    assert abs(hit.mean() - p_scatter.mean()) < 0.01
    depth = (h["t"][hit] - entry[hit])
    # mean of the truncated exponential on [0, 2]
    lam = 0.7
    tm = (1.0 / lam - 2.0 * math.exp(-2 * lam) / (1 - math.exp(-2 * lam)))
    assert abs(depth.mean() - tm) < 0.02
