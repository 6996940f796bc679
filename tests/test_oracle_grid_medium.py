"""The voxel-grid medium of the CPU oracle (no counterpart in the reference):
σ_t = density × trilinear(grid) in a box, delta tracking against per-brick
majorants for the scatter distance and ratio tracking for shadow
transmittance.  Both are checked against the optical depth integrated here
in float64: the transmittance estimator is unbiased, the scatter probability
is 1 − exp(−τ) and the optical depth at the scatter point follows the
truncated exponential law."""
import math

import numpy as np

from oracle import oracle as O
from rustracer_b200.scene import SceneBuilder

LO = np.array([0.0, 0.0, 0.0])
HI = np.array([1.0, 0.5, 1.0])


def grid_scene(grid, density):
    sb = SceneBuilder()
    sb.add_medium("grid", "box", density, (0.9, 0.9, 0.9), g=0.3, p_min=tuple(LO), p_max=tuple(HI), grid=grid)
    return sb


def sigma(grid, density, p):
    """σ_t at points p (n, 3): trilinear between voxel centres, clamped (float64)."""
    nz, ny, nx = grid.shape
    res = np.array([nx, ny, nz], np.float64)
    c = (p - LO) / (HI - LO) * res - 0.5
    u = np.clip(c, 0.0, res - 1)
    i0 = np.minimum(np.floor(u).astype(int), np.maximum(res.astype(int) - 2, 0))
    i1 = np.minimum(i0 + 1, res.astype(int) - 1)
    f = u - i0
    g = grid.astype(np.float64)
    out = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                ix = i1[:, 0] if dx else i0[:, 0]
                iy = i1[:, 1] if dy else i0[:, 1]
                iz = i1[:, 2] if dz else i0[:, 2]
                w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1]) * (f[:, 2] if dz else 1 - f[:, 2])
                out = out + w * g[iz, iy, ix]
    return density * out


def box_interval(o, d):
    inv = 1.0 / d
    t0, t1 = (LO - o) * inv, (HI - o) * inv
    return np.max(np.minimum(t0, t1)), np.min(np.maximum(t0, t1))


def optical_depth(grid, density, o, d, a, b, n=40001):
    t = np.linspace(a, b, n)
    s = sigma(grid, density, o[None] + t[:, None] * d[None])
    return np.trapezoid(s, t) * np.linalg.norm(d), t, s


def _grid(seed, shape=(16, 12, 20), zero_slab=True):
    rng = np.random.default_rng(seed)
    g = rng.gamma(1.5, 0.5, size=shape).astype(np.float32)
    if zero_slab:
        g[:, :, 5:9] = 0.0          # empty bricks along x: the walk must skip them
    return g


def _rays(o, d, n, tmax=np.inf, seed=0):
    """n copies of one ray whose origins differ in the last bits (each its own
    random stream, the same segment to within 1e-6)."""
    rng = np.random.default_rng(seed)
    oo = np.tile(o, (n, 1)) + rng.uniform(-1e-6, 1e-6, (n, 3))
    return np.concatenate([oo, np.tile(d, (n, 1)), np.full((n, 1), 0.001), np.full((n, 1), tmax)], 1).astype(np.float32)


def test_ratio_tracking_transmittance_is_unbiased():
    grid = _grid(1)
    s = O.OracleScene(grid_scene(grid, 3.0))
    for o, d, tmax in [((-1.0, 0.25, 0.31), (1.0, 0.02, 0.05), np.inf),
                       ((0.5, -0.5, 0.5), (0.1, 1.0, -0.2), np.inf),
                       ((0.1, 0.1, 0.9), (0.7, 0.15, -0.6), 0.8)]:
        o, d = np.array(o), np.array(d)
        a, b = box_interval(o, d)
        a, b = max(a, 0.001), min(b, tmax)
        tau = optical_depth(grid, 3.0, o, d, a, b)[0]
        tr = s.trace_transmittance(_rays(o, d, 20000, tmax, seed=2))
        assert (tr >= 0).all() and (tr <= 1).all()
        se = tr.std() / math.sqrt(len(tr))
        assert abs(tr.mean() - math.exp(-tau)) < 4 * se + 1e-4, (tr.mean(), math.exp(-tau), se)


def test_delta_tracking_scatter_law():
    grid = _grid(3)
    density = 2.5
    s = O.OracleScene(grid_scene(grid, density))
    o, d = np.array([-0.5, 0.2, 0.4]), np.array([1.0, 0.05, 0.1])
    a, b = box_interval(o, d)
    tau, ts, ss = optical_depth(grid, density, o, d, a, b)
    n = 40000
    h = s.trace_closest(_rays(o, d, n, seed=4))
    hit = h["prim"] == 0                               # the medium's id: there are no primitives
    p = 1.0 - math.exp(-tau)
    assert abs(hit.mean() - p) < 4 * math.sqrt(p * (1 - p) / n), (hit.mean(), p)
    # optical depth up to each scatter point: exponential truncated at τ
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (ss[1:] + ss[:-1]) * np.diff(ts))]) * np.linalg.norm(d)
    tau_s = np.interp(h["t"][hit].astype(np.float64), ts, cum)
    mean = 1.0 - tau * math.exp(-tau) / (1.0 - math.exp(-tau))
    assert abs(tau_s.mean() - mean) < 4 * tau_s.std() / math.sqrt(hit.sum())
    # no scatter point in the empty slab
    x = o[0] + h["t"][hit] * d[0]
    assert not ((x > 5.6 / 20) & (x < 8.4 / 20)).any()      # σ_t = 0 between the zero voxels' centres


def test_grid_medium_needs_a_box_and_valid_voxels():
    import pytest
    sb = SceneBuilder()
    with pytest.raises(ValueError):
        sb.add_medium("grid", "sphere", 1.0, (1, 1, 1), center=(0, 0, 0), radius=1.0, grid=np.ones((2, 2, 2)))
    bad = np.ones((4, 4, 4), np.float32)
    bad[1, 1, 1] = -1.0
    with pytest.raises(Exception):
        O.OracleScene(grid_scene(bad, 1.0))
